// rs_pybind.cpp -- pybind11 module `ropesim._ropesim`: RopeSim, RopeBatch and CudaView with the
// signatures, defaults and ValueError validation of the reference's bindings
// (csrc/bindings.cpp:629-1210), implemented on the C-ABI of include/ropesim_b200.h. Device
// arrays arrive through __cuda_array_interface__ (torch, cupy, numba); torch itself is not a
// dependency of this module.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ropesim_b200.h"

namespace py = pybind11;
static_assert(sizeof(rs_backward_io) == 28 * sizeof(const float*), "rs_backward_io is 28 pointers");
static_assert(sizeof(rs_frame_io) == 16 * sizeof(const float*), "rs_frame_io is 16 pointers");
using farray = py::array_t<float, py::array::c_style | py::array::forcecast>;

namespace {

// C-ABI status -> Python exception (RS_EINVAL -> ValueError, others -> RuntimeError).
void ok(int rc) {
    if (rc == RS_OK) return;
    const std::string msg = rs_last_error_string();
    if (rc == RS_EINVAL) throw py::value_error(msg);
    throw std::runtime_error(msg);
}

std::vector<float> vec3(const farray& a, const char* name) {
    if (a.ndim() != 1 || a.shape(0) != 3) throw py::value_error(std::string(name) + " must be a length-3 array");
    return {a.data()[0], a.data()[1], a.data()[2]};
}

// A float32, C-contiguous CUDA array of exactly `want` (bindings.cpp:587-617).
uintptr_t parse_cai(const py::object& obj, const std::vector<py::ssize_t>& want, const char* name) {
    if (!py::hasattr(obj, "__cuda_array_interface__"))
        throw py::value_error(std::string(name) + " must be a CUDA array (e.g. a contiguous float32 torch tensor on cuda)");
    py::dict d = obj.attr("__cuda_array_interface__").cast<py::dict>();
    const auto ts = d["typestr"].cast<std::string>();
    if (ts != "<f4") throw py::value_error(std::string(name) + " must be float32 (got " + ts + ")");
    auto shape = d["shape"].cast<std::vector<py::ssize_t>>();
    if (shape != want) {
        std::string s = std::string(name) + " has wrong shape; expected (";
        for (auto v : want) s += std::to_string(v) + ",";
        throw py::value_error(s + ")");
    }
    py::object st = d.attr("get")("strides", py::none());
    if (!st.is_none()) {
        auto strides = st.cast<std::vector<py::ssize_t>>();
        py::ssize_t expect = 4;
        for (size_t i = shape.size(); i-- > 0;) {
            if (shape[i] != 1 && strides[i] != expect) throw py::value_error(std::string(name) + " must be C-contiguous");
            expect *= shape[i];
        }
    }
    return d["data"].cast<py::tuple>()[0].cast<uintptr_t>();
}

// A per-vertex CUDA array of k components (k = 0: scalar per vertex) in caller order, as
// [total_verts(, k)] or, for equal-length ropes, [num_envs, V(, k)]. None -> 0.
uintptr_t parse_vertex_array(const py::object& obj, int n, int R, int V, int k, const char* name) {
    if (obj.is_none()) return 0;
    if (!py::hasattr(obj, "__cuda_array_interface__"))
        throw py::value_error(std::string(name) + " must be a CUDA array (e.g. a contiguous float32 torch tensor on cuda)");
    auto shape = obj.attr("__cuda_array_interface__").cast<py::dict>()["shape"].cast<std::vector<py::ssize_t>>();
    std::vector<py::ssize_t> flat{n}, grid{R, V};
    if (k > 0) { flat.push_back(k); grid.push_back(k); }
    return parse_cai(obj, (V > 0 && shape.size() == grid.size()) ? grid : flat, name);
}

// Device buffer handed back to Python; torch.as_tensor(view) shares it (bindings.cpp:622-625).
struct CudaView {
    uintptr_t ptr;
    std::vector<py::ssize_t> shape;
};

void validate_rows(const float* p, const float* q, int rows, const char* who) {
    for (int r = 0; r < rows; r++) {
        const float l = std::sqrt(q[4 * r] * q[4 * r] + q[4 * r + 1] * q[4 * r + 1] + q[4 * r + 2] * q[4 * r + 2] + q[4 * r + 3] * q[4 * r + 3]);
        if (!std::isfinite(l) || !(l > 1e-6f)) throw py::value_error(std::string(who) + ": quat must be finite with nonzero norm");
        if (!std::isfinite(p[3 * r]) || !std::isfinite(p[3 * r + 1]) || !std::isfinite(p[3 * r + 2]))
            throw py::value_error(std::string(who) + ": pos must be finite");
    }
}
int parse_poses(const farray& pos, const farray& quat, int N, const char* who) {
    const bool p1 = pos.ndim() == 1 && pos.shape(0) == 3, pN = pos.ndim() == 2 && pos.shape(0) == N && pos.shape(1) == 3;
    const bool q1 = quat.ndim() == 1 && quat.shape(0) == 4, qN = quat.ndim() == 2 && quat.shape(0) == N && quat.shape(1) == 4;
    if (!((p1 && q1) || (pN && qN)))
        throw py::value_error(std::string(who) + ": pos must be [3] and quat [4] (x, y, z, w), or [num_envs, 3] and [num_envs, 4]");
    const int rows = p1 ? 1 : N;
    validate_rows(pos.data(), quat.data(), rows, who);
    return rows;
}

struct Tele {
    bool all = false, device = false;
    const uint8_t* ptr = nullptr;
    std::vector<uint8_t> host;
};
Tele parse_teleport(const py::object& teleport, int N, const char* who) {
    Tele t;
    if (py::isinstance<py::bool_>(teleport)) { t.all = teleport.cast<bool>(); return t; }
    if (py::hasattr(teleport, "__cuda_array_interface__")) {
        py::dict d = teleport.attr("__cuda_array_interface__").cast<py::dict>();
        const auto ts = d["typestr"].cast<std::string>();
        auto shape = d["shape"].cast<std::vector<py::ssize_t>>();
        py::object st = d.attr("get")("strides", py::none());
        const bool contiguous = st.is_none() || N == 1 || st.cast<std::vector<py::ssize_t>>() == std::vector<py::ssize_t>{1};
        if ((ts != "|b1" && ts != "|u1") || shape != std::vector<py::ssize_t>{N} || !contiguous)
            throw py::value_error(std::string(who) + ": teleport must be a bool, a [num_envs] bool array, or a contiguous [num_envs] CUDA bool array");
        t.device = true;
        t.ptr = reinterpret_cast<const uint8_t*>(d["data"].cast<py::tuple>()[0].cast<uintptr_t>());
        return t;
    }
    auto a = py::array_t<bool, py::array::c_style | py::array::forcecast>::ensure(teleport);
    if (!a || a.ndim() != 1 || a.shape(0) != N)
        throw py::value_error(std::string(who) + ": teleport must be a bool, a [num_envs] bool array, or a [num_envs] CUDA bool array");
    t.host.resize(N);
    for (int i = 0; i < N; i++) t.host[i] = a.data()[i] ? 1 : 0;
    t.ptr = t.host.data();
    return t;
}

float mu_or(const py::object& mu, float dflt) { return mu.is_none() ? dflt : mu.cast<float>(); }

// The shared engine handle: one rs_batch per Python object.
class Engine {
public:
    rs_batch* h = nullptr;
    int n = 0, R = 0;
    ~Engine() {
        if (h) rs_batch_destroy(h);
    }
    float get(int which) const {
        float v = 0.f;
        ok(rs_batch_get_param(h, which, &v));
        return v;
    }
    void set(int which, float v) { ok(rs_batch_set_param(h, which, v)); }
    void set_planes(const farray& planes, float radius, float mu_s, py::object mu_k, float v_slip, float kappa) {
        if (planes.ndim() != 2 || planes.shape(1) != 4 || planes.shape(0) > 8)
            throw py::value_error("planes must be [P<=8, 4] rows (nx, ny, nz, w): half-spaces n.x >= w");
        const int P = (int)planes.shape(0);
        const float mk = mu_k.is_none() ? mu_s : mu_k.cast<float>();
        if (P > 0 && (!(radius > 0) || !(kappa > 0) || !(mu_s >= 0) || !(mk >= 0) || !(v_slip > 0)))
            throw py::value_error("plane contact needs radius > 0, kappa > 0, mu_s >= 0, mu_k >= 0, v_slip > 0");
        for (int i = 0; i < P; i++) {
            const float* r = planes.data() + 4 * i;
            const float l = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (!(l > 0) || !std::isfinite(l) || !std::isfinite(r[3]))
                throw py::value_error("plane rows need a finite, nonzero normal and a finite offset");
        }
        ok(rs_batch_set_planes(h, P, planes.data()));
        if (P > 0) ok(rs_batch_set_contact(h, radius, mu_s, mk, v_slip, kappa));
    }
    void set_contact(float radius, float mu_s, py::object mu_k, float v_slip, float kappa) {
        ok(rs_batch_set_contact(h, radius, mu_s, mu_k.is_none() ? mu_s : mu_k.cast<float>(), v_slip, kappa));
    }
    int add_mesh(const farray& values, const farray& origin, float spacing, const farray& pos, const farray& quat,
                 py::object mu_s, py::object mu_k, int N) {
        if (values.ndim() != 3 || values.shape(0) < 2 || values.shape(1) < 2 || values.shape(2) < 2)
            throw py::value_error("sdf values must be [nx, ny, nz] with every dim >= 2");
        if (!(spacing > 0) || !std::isfinite(spacing)) throw py::value_error("sdf spacing must be > 0");
        const auto o = vec3(origin, "origin");
        const int rows = parse_poses(pos, quat, N, "add_mesh");
        float r = 0.f, ms0 = 0.f, mk0 = 0.f;
        ok(rs_batch_get_contact(h, &r, &ms0, &mk0));
        if (!(r > 0)) throw py::value_error("set the contact material first: set_contact(radius, ...) or set_planes(..., radius=)");
        const float ms = mu_or(mu_s, ms0), mk = mu_or(mu_k, mu_s.is_none() ? mk0 : ms);
        if (!(ms >= 0) || !(mk >= 0)) throw py::value_error("mu_s / mu_k must be >= 0");
        int idx = -1;
        {
            py::gil_scoped_release rel;
            ok(rs_batch_add_mesh(h, values.data(), (int)values.shape(0), (int)values.shape(1), (int)values.shape(2), o.data(),
                                 spacing, ms, mk, pos.data(), quat.data(), rows, &idx));
        }
        return idx;
    }
    void set_mesh_friction(int index, float mu_s, py::object mu_k) {
        if (!(mu_s >= 0)) throw py::value_error("mu_s must be >= 0");
        const float mk = mu_or(mu_k, mu_s);
        if (!(mk >= 0)) throw py::value_error("mu_k must be >= 0");
        ok(rs_batch_set_mesh_friction(h, index, mu_s, mk));
    }
    int meshes() const {
        int m = 0;
        ok(rs_batch_num_meshes(h, &m));
        return m;
    }
};

py::array_t<float> arr2(int rows, int cols) { return py::array_t<float>({(py::ssize_t)rows, (py::ssize_t)cols}); }

// ------------------------------------------------------------------ RopeSim (bindings.cpp:185-582)
class RopeSim : public Engine {
public:
    bool collisions = false, fixRoot = false;
    RopeSim(int num_verts, float seg_len, const farray& dir, float density, float k_stretch, float k_bend, float max_h,
            int num_itr, bool fix_root_orientation, bool collisions_) {
        if (num_verts < 3) throw py::value_error("num_verts must be >= 3");
        if (!(seg_len > 0)) throw py::value_error("seg_len must be > 0");
        if (!(density > 0)) throw py::value_error("density must be > 0");
        if (!(k_stretch > 0)) throw py::value_error("k_stretch must be > 0");
        if (!(k_bend > 0))
            throw py::value_error("k_bend must be > 0: k_bend=0 zeroes the rest-frame vectors and the orientation solve "
                                  "produces NaNs (normalize of a zero vector)");
        if (!(max_h > 0)) throw py::value_error("max_h must be > 0");
        if (num_itr < 1) throw py::value_error("num_itr must be >= 1");
        auto d = vec3(dir, "dir");
        const float dl = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (!(dl > 0)) throw py::value_error("dir must be nonzero");
        if (collisions_ && 2 * seg_len < 2 * 1e-4f + 8e-4f)
            throw py::value_error("collisions=True uses the upstream yarn-scale collision radius (1e-4 m): seg_len must be >= 5e-4 m");
        collisions = collisions_;
        fixRoot = fix_root_orientation;
        // vertex i at i * seg_len * (dir / |dir|), bindings.cpp:217-219
        std::vector<float> pos(3 * (size_t)num_verts);
        for (int i = 0; i < num_verts; i++)
            for (int k = 0; k < 3; k++) pos[3 * i + k] = float(i) * seg_len * (d[k] / dl);
        const int verts = num_verts;
        // collisions=True keeps YarnBall's yarn-scale radius/barrier (YarnBall.cu:33-34), else the
        // dead radii scale with the segment (bindings.cpp:225-244)
        const float rad = collisions_ ? 1e-4f : 0.01f * seg_len, bar = collisions_ ? 8e-4f : 0.08f * seg_len;
        ok(rs_batch_create(&h, 1, &verts, pos.data(), nullptr, density, k_stretch, k_bend, max_h, num_itr,
                           fix_root_orientation ? 1 : 0, 0, rad, bar));
        n = num_verts;
        R = 1;
        // self contact of the rope through the rope-rope path with YarnBall's defaults
        // (kCollision 1e-5, friction 0.1, kFriction 5, detection scaler 1.2; YarnBall.cu:37-40)
        if (collisions_) ok(rs_batch_set_rope_contact(h, 1, 1e-4f, 8e-4f, 1e-5f, 0.1f, 5.f, 1.2f, 1));
    }
    void advance(float dt, int substeps) {
        if (substeps < 0) throw py::value_error("substeps must be >= 0");
        if (!(dt > 0)) return;
        py::gil_scoped_release rel;
        ok(rs_batch_advance(h, dt, substeps));
    }
    void set_root(const farray& pos, const farray& vel, py::object q) {
        const auto p = vec3(pos, "pos"), v = vec3(vel, "vel");
        std::vector<float> qq;
        if (!q.is_none()) {
            if (!fixRoot) throw py::value_error("set_root(q=...) requires fix_root_orientation=True");
            farray qa = q.cast<farray>();
            if (qa.ndim() != 1 || qa.shape(0) != 4) throw py::value_error("q must be a length-4 array (x,y,z,w)");
            const float* b = qa.data();
            const float l = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2] + b[3] * b[3]);
            if (!std::isfinite(l) || !(l > 1e-6f)) throw py::value_error("q must be finite with nonzero norm");
            qq = {b[0] / l, b[1] / l, b[2] / l, b[3] / l};
        }
        std::vector<float> im(n);
        ok(rs_batch_inv_masses(h, im.data()));
        if (im[0] != 0.f) throw py::value_error("set_root drives a pinned root; this rope's root was unpinned (unpin_root)");
        ok(rs_batch_set_root(h, 0, p.data(), v.data(), qq.empty() ? nullptr : qq.data()));
    }
    py::array_t<float> positions() {
        auto a = arr2(n, 3);
        ok(rs_batch_download(h, a.mutable_data(), nullptr, nullptr));
        return a;
    }
    py::array_t<float> velocities() {
        auto a = arr2(n, 3);
        ok(rs_batch_download(h, nullptr, a.mutable_data(), nullptr));
        return a;
    }
    py::array_t<float> quaternions() {
        auto a = arr2(n, 4);
        ok(rs_batch_download(h, nullptr, nullptr, a.mutable_data()));
        return a;
    }
    py::array_t<float> inv_masses() {
        py::array_t<float> a(n);
        ok(rs_batch_inv_masses(h, a.mutable_data()));
        return a;
    }
    py::array_t<float> rest_lengths() {
        std::vector<float> all(n);
        ok(rs_batch_rest_lengths(h, all.data()));
        py::array_t<float> a(n - 1);
        for (int i = 0; i < n - 1; i++) a.mutable_data()[i] = all[i];
        return a;
    }
    void set_stiff(const farray& a, bool stretch) {
        if (a.ndim() != 1 || a.shape(0) != n - 1)
            throw py::value_error(stretch ? "expected length n-1 array of EA values" : "expected length n-1 array of EI values");
        for (int i = 0; i < n - 1; i++)
            if (!std::isfinite(a.data()[i]) || !(a.data()[i] > 0))
                throw py::value_error(stretch ? "EA values must be finite and > 0" : "EI values must be finite and > 0");
        std::vector<float> full(n, 1.f);
        for (int i = 0; i < n - 1; i++) full[i] = a.data()[i];
        ok(stretch ? rs_batch_set_stretch_stiffnesses(h, full.data()) : rs_batch_set_bend_stiffnesses(h, full.data()));
    }
    void set_velocities(const farray& v) {
        if (v.ndim() != 2 || v.shape(0) != n || v.shape(1) != 3) throw py::value_error("expected [n,3] array of velocities");
        ok(rs_batch_set_velocities(h, v.data()));
    }
    void set_mesh_pose(int index, const farray& pos, const farray& quat, bool teleport) {
        parse_poses(pos, quat, 1, "set_mesh_pose");
        ok(rs_batch_set_mesh_poses(h, index, pos.data(), quat.data(), 1, nullptr, teleport ? 1 : 0, 0));
    }
    py::array_t<float> contact_forces() {
        auto a = arr2(n, 3);
        ok(rs_batch_contact_forces(h, a.mutable_data()));
        return a;
    }
    py::array_t<float> mesh_wrenches() {
        auto a = arr2(meshes(), 6);
        ok(rs_batch_mesh_wrenches(h, a.mutable_data()));
        return a;
    }
};

// ------------------------------------------------------------------ RopeBatch (bindings.cpp:735-1210)
class RopeBatch : public Engine {
public:
    int V = 0;           // verts per rope (uniform batches)
    bool fixRoot = false;
    bool stepped = false;
    bool rootsPinned = true;
    std::vector<int> verts;

    std::vector<py::ssize_t> vshape(int k) const {
        if (V > 0) return {R, V, k};
        return {n, k};
    }
    void step(py::object root_pos, py::object root_vel, float dt, int substeps, py::object root_q, py::object root_pos_end,
              py::object root_q_end) {
        if (!(dt > 0)) throw py::value_error("dt must be > 0");
        if (substeps < 1) throw py::value_error("substeps must be >= 1");
        if (!rootsPinned)
            throw py::value_error("step() drives every rope's root; ropes built with a free root (from_positions pinned=...) advance with step_free()");
        const uintptr_t p = parse_cai(root_pos, {R, 3}, "root_pos");
        const uintptr_t v = parse_cai(root_vel, {R, 3}, "root_vel");
        uintptr_t q = 0;
        if (!root_q.is_none()) {
            if (!fixRoot) throw py::value_error("root_q requires fix_root_orientation=True");
            q = parse_cai(root_q, {R, 4}, "root_q");
        }
        if (root_pos_end.is_none()) {
            if (!root_q_end.is_none()) throw py::value_error("root_q_end requires root_pos_end (the motion-program path)");
            stepped = true;
            py::gil_scoped_release rel;
            ok(rs_batch_step_legacy(h, (const float*)p, (const float*)v, (const float*)q, dt, substeps, 0));
            return;
        }
        const uintptr_t p1 = parse_cai(root_pos_end, {R, 3}, "root_pos_end");
        uintptr_t q1 = 0;
        if (!root_q_end.is_none()) {
            if (q == 0) throw py::value_error("root_q_end requires root_q");
            q1 = parse_cai(root_q_end, {R, 4}, "root_q_end");
        }
        stepped = true;
        py::gil_scoped_release rel;
        ok(rs_batch_step_program(h, (const float*)p, (const float*)v, (const float*)p1, (const float*)q, (const float*)q1, dt,
                                 substeps, 0));
    }
    // Per-vertex arrays broadcast from [V-ish] or [N, V-ish] (bindings.cpp:1121-1201).
    std::vector<float> per_vertex(const farray& a, int cols_minus, const char* msg) {
        const bool per_env = a.ndim() == 2;
        if (V == 0) {
            if (!(a.ndim() == 1 && a.shape(0) == n)) throw py::value_error(std::string(msg) + " (flat [total_verts] for uneven ropes)");
            return std::vector<float>(a.data(), a.data() + n);
        }
        const int C = V - cols_minus;
        if (!((a.ndim() == 1 && a.shape(0) == C) || (per_env && a.shape(0) == R && a.shape(1) == C))) throw py::value_error(msg);
        std::vector<float> out((size_t)n, 1.f);
        for (int e = 0; e < R; e++)
            for (int v = 0; v < C; v++) out[(size_t)e * V + v] = per_env ? a.data()[(size_t)e * C + v] : a.data()[v];
        return out;
    }
};

std::unique_ptr<RopeBatch> make_batch(int N, const std::vector<int>& verts, const float* pos, const uint8_t* pin,
                                      float density, float ks, float kb, float max_h, int num_itr, bool fix_root,
                                      bool straight_rest, float minSeg) {
    auto b = std::make_unique<RopeBatch>();
    ok(rs_batch_create(&b->h, N, verts.data(), pos, pin, density, ks, kb, max_h, num_itr, fix_root ? 1 : 0,
                       straight_rest ? 1 : 0, 0.01f * minSeg, 0.08f * minSeg));
    b->R = N;
    b->verts = verts;
    b->n = 0;
    for (int v : verts) b->n += v;
    bool uni = true;
    for (int v : verts) uni = uni && v == verts[0];
    b->V = uni ? verts[0] : 0;
    b->fixRoot = fix_root;
    int rp = 1;
    ok(rs_batch_roots_pinned(b->h, &rp));
    b->rootsPinned = rp != 0;
    return b;
}

}  // namespace

#ifndef RS_MODULE_NAME
#define RS_MODULE_NAME _ropesim
#endif
PYBIND11_MODULE(RS_MODULE_NAME, m) {
    m.doc() = "B200 Stable Cosserat Rods engine (persistent sm_100a frame kernel) behind the ropesim API";
    m.attr("__version__") = rs_version();

    // the GPU half of ropesim.sdf.bake_mesh (lattice box and closedness checks are in Python)
    m.def("bake_sdf",
          [](farray vertices, py::array_t<int, py::array::c_style | py::array::forcecast> triangles, farray origin,
             double spacing, std::vector<int> dims, float thickness, float round, bool counters) {
              if (vertices.ndim() != 2 || vertices.shape(1) != 3) throw py::value_error("vertices must be [V, 3]");
              if (triangles.ndim() != 2 || triangles.shape(1) != 3) throw py::value_error("triangles must be [T, 3]");
              if (dims.size() != 3) throw py::value_error("dims must be (nx, ny, nz)");
              const auto o = vec3(origin, "origin");
              py::array_t<float> out({(py::ssize_t)dims[0], (py::ssize_t)dims[1], (py::ssize_t)dims[2]});
              unsigned long long cnt[4] = {0, 0, 0, 0};
              const float* vp = vertices.data();
              const int* tp = triangles.data();
              float* op = out.mutable_data();
              const int nv = (int)vertices.shape(0), nt = (int)triangles.shape(0);
              int rc;
              {
                  py::gil_scoped_release nogil;
                  rc = rs_sdf_bake(vp, nv, tp, nt, o.data(), spacing, dims[0], dims[1], dims[2], thickness, round, op, 0,
                                   nullptr, counters ? cnt : nullptr);
              }
              ok(rc);
              if (!counters) return py::object(out);
              return py::object(py::make_tuple(out, cnt[0], cnt[1], cnt[2]));
          },
          py::arg("vertices"), py::arg("triangles"), py::arg("origin"), py::arg("spacing"), py::arg("dims"),
          py::arg("thickness") = 0.f, py::arg("round") = 0.f, py::arg("counters") = false);

    py::class_<CudaView>(m, "CudaView")
        .def_property_readonly("__cuda_array_interface__", [](const CudaView& v) {
            py::dict d;
            py::tuple shape(v.shape.size());
            for (size_t i = 0; i < v.shape.size(); i++) shape[i] = v.shape[i];
            d["shape"] = shape;
            d["typestr"] = "<f4";
            d["data"] = py::make_tuple(v.ptr, false);
            d["strides"] = py::none();
            d["version"] = 2;
            return d;
        })
        .def_property_readonly("ptr", [](const CudaView& v) { return v.ptr; })
        .def_property_readonly("shape", [](const CudaView& v) {
            py::tuple t(v.shape.size());
            for (size_t i = 0; i < v.shape.size(); i++) t[i] = v.shape[i];
            return t;
        });

    py::class_<RopeSim>(m, "RopeSim")
        .def(py::init([](int num_verts, float seg_len, farray dir, float density, float k_stretch, float k_bend, float max_h,
                         int num_itr, bool fix_root_orientation, bool collisions) {
                 return new RopeSim(num_verts, seg_len, dir, density, k_stretch, k_bend, max_h, num_itr, fix_root_orientation,
                                    collisions);
             }),
             py::arg("num_verts"), py::arg("seg_len") = 0.02f, py::arg("dir") = farray(py::cast(std::vector<float>{1, 0, 0})),
             py::arg("density") = 0.1f, py::arg("k_stretch") = 500.0f, py::arg("k_bend") = 1e-6f,
             py::arg("max_h") = 1.f / 3000.f, py::arg("num_itr") = 8, py::arg("fix_root_orientation") = false,
             py::arg("collisions") = false)
        .def("advance", &RopeSim::advance, py::arg("dt"), py::arg("substeps") = 0)
        .def("reset", [](RopeSim& s) { ok(rs_batch_reset_all(s.h)); })
        .def("set_root", &RopeSim::set_root, py::arg("pos"), py::arg("vel"), py::arg("q") = py::none())
        .def("positions", &RopeSim::positions)
        .def("velocities", &RopeSim::velocities)
        .def("quaternions", &RopeSim::quaternions)
        .def("inv_masses", &RopeSim::inv_masses)
        .def("rest_lengths", &RopeSim::rest_lengths)
        .def("set_stretch_stiffnesses", [](RopeSim& s, farray a) { s.set_stiff(a, true); }, py::arg("ea"))
        .def("set_bend_stiffnesses", [](RopeSim& s, farray a) { s.set_stiff(a, false); }, py::arg("ei"))
        .def("set_gravity", [](RopeSim& s, farray g) { ok(rs_batch_set_gravity(s.h, vec3(g, "gravity").data())); }, py::arg("gravity"))
        .def("set_planes", &RopeSim::set_planes, py::arg("planes"), py::arg("radius") = 0.f, py::arg("mu_s") = 0.5f,
             py::arg("mu_k") = py::none(), py::arg("v_slip") = 1e-3f, py::arg("kappa") = 2.f)
        .def("unpin_root", [](RopeSim& s) { ok(rs_batch_unpin_root(s.h, 0)); })
        .def("set_contact", &RopeSim::set_contact, py::arg("radius"), py::arg("mu_s") = 0.5f, py::arg("mu_k") = py::none(),
             py::arg("v_slip") = 1e-3f, py::arg("kappa") = 2.f)
        .def("add_mesh",
             [](RopeSim& s, farray values, farray origin, float spacing, farray pos, farray quat, py::object mu_s,
                py::object mu_k) { return s.add_mesh(values, origin, spacing, pos, quat, mu_s, mu_k, 1); },
             py::arg("values"), py::arg("origin"), py::arg("spacing"),
             py::arg("pos") = farray(py::cast(std::vector<float>{0, 0, 0})),
             py::arg("quat") = farray(py::cast(std::vector<float>{0, 0, 0, 1})), py::arg("mu_s") = py::none(),
             py::arg("mu_k") = py::none())
        .def("set_mesh_friction", &RopeSim::set_mesh_friction, py::arg("index"), py::arg("mu_s"), py::arg("mu_k") = py::none())
        .def("set_mesh_pose", &RopeSim::set_mesh_pose, py::arg("index"), py::arg("pos"), py::arg("quat"), py::arg("teleport") = false)
        .def("clear_meshes", [](RopeSim& s) { ok(rs_batch_clear_meshes(s.h)); })
        .def("enable_contact_forces", [](RopeSim& s, bool on) { ok(rs_batch_enable_contact_forces(s.h, on ? 1 : 0)); },
             py::arg("on") = true)
        .def("contact_forces", &RopeSim::contact_forces)
        .def("mesh_wrenches", &RopeSim::mesh_wrenches)
        .def_property("drag", [](RopeSim& s) { return s.get(RS_P_DRAG); }, [](RopeSim& s, float v) { s.set(RS_P_DRAG, v); })
        .def_property("drag_quad", [](RopeSim& s) { return s.get(RS_P_DRAG_QUAD); },
                      [](RopeSim& s, float v) { s.set(RS_P_DRAG_QUAD, v); })
        .def_property("drag_quad_t", [](RopeSim& s) { return s.get(RS_P_DRAG_QUAD_T); },
                      [](RopeSim& s, float v) { s.set(RS_P_DRAG_QUAD_T, v); })
        .def("set_velocities", &RopeSim::set_velocities, py::arg("velocities"))
        .def_property("damping", [](RopeSim& s) { return s.get(RS_P_DAMPING); }, [](RopeSim& s, float v) { s.set(RS_P_DAMPING, v); })
        .def_property("num_itr", [](RopeSim& s) { int v; ok(rs_batch_get_num_itr(s.h, &v)); return v; },
                      [](RopeSim& s, int v) {
                          if (v < 1) throw py::value_error("num_itr must be >= 1");
                          ok(rs_batch_set_num_itr(s.h, v));
                      })
        .def_property("accel_ratio", [](RopeSim& s) { return s.get(RS_P_ACCEL); }, [](RopeSim& s, float v) { s.set(RS_P_ACCEL, v); })
        .def_property("max_h", [](RopeSim& s) { return s.get(RS_P_MAX_H); },
                      [](RopeSim& s, float v) {
                          if (!(v > 0)) throw py::value_error("max_h must be > 0");
                          s.set(RS_P_MAX_H, v);
                      })
        .def_property_readonly("gravity", [](RopeSim& s) {
            py::array_t<float> a(3);
            ok(rs_batch_get_gravity(s.h, a.mutable_data()));
            return a;
        })
        .def_property_readonly("time", [](RopeSim& s) { return s.get(RS_P_TIME); })
        .def_property_readonly("last_error", [](RopeSim& s) { int e; ok(rs_batch_status(s.h, &e, nullptr, nullptr)); return e; })
        .def_property_readonly("last_warning", [](RopeSim& s) { int w; ok(rs_batch_status(s.h, nullptr, &w, nullptr)); return w; })
        .def_property_readonly("collisions_enabled", [](RopeSim& s) { return s.collisions; })
        .def_property_readonly("fixed_root_orientation", [](RopeSim& s) { return s.fixRoot; })
        .def_property_readonly("num_verts", [](RopeSim& s) { return s.n; });

    py::class_<RopeBatch>(m, "RopeBatch")
        .def(py::init([](int num_envs, int verts_per_rope, farray root_pos, float seg_len, farray dir, float density,
                         float k_stretch, float k_bend, float max_h, int num_itr, bool fix_root_orientation, bool deterministic) {
                 (void)deterministic;  // sweeps are always the deterministic (Jacobi) ordering here
                 if (num_envs < 1) throw py::value_error("num_envs must be >= 1");
                 if (verts_per_rope < 3) throw py::value_error("verts_per_rope must be >= 3");
                 if (!(seg_len > 0)) throw py::value_error("seg_len must be > 0");
                 if (!(density > 0)) throw py::value_error("density must be > 0");
                 if (!(k_stretch > 0)) throw py::value_error("k_stretch must be > 0");
                 if (!(k_bend > 0)) throw py::value_error("k_bend must be > 0 (0 -> NaN, see RopeSim)");
                 if (!(max_h > 0)) throw py::value_error("max_h must be > 0");
                 if (num_itr < 1) throw py::value_error("num_itr must be >= 1");
                 if (root_pos.ndim() != 2 || root_pos.shape(0) != num_envs || root_pos.shape(1) != 3)
                     throw py::value_error("root_pos must be a host [num_envs, 3] array");
                 const auto d = vec3(dir, "dir");
                 if (!(std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) > 0)) throw py::value_error("dir must be nonzero");
                 auto b = std::make_unique<RopeBatch>();
                 ok(rs_batch_create_straight(&b->h, num_envs, verts_per_rope, root_pos.data(), seg_len, d.data(), density,
                                             k_stretch, k_bend, max_h, num_itr, fix_root_orientation ? 1 : 0,
                                             0.01f * seg_len, 0.08f * seg_len));
                 b->R = num_envs;
                 b->V = verts_per_rope;
                 b->n = num_envs * verts_per_rope;
                 b->verts.assign(num_envs, verts_per_rope);
                 b->fixRoot = fix_root_orientation;
                 return b.release();
             }),
             py::arg("num_envs"), py::arg("verts_per_rope"), py::arg("root_pos"), py::arg("seg_len") = 0.02f,
             py::arg("dir") = farray(py::cast(std::vector<float>{0, 0, -1})), py::arg("density") = 0.1f,
             py::arg("k_stretch") = 500.0f, py::arg("k_bend") = 1e-6f, py::arg("max_h") = 1.f / 3000.f,
             py::arg("num_itr") = 8, py::arg("fix_root_orientation") = true, py::arg("deterministic") = false)
        .def("step", &RopeBatch::step, py::arg("root_pos"), py::arg("root_vel"), py::arg("dt"), py::arg("substeps"),
             py::arg("root_q") = py::none(), py::arg("root_pos_end") = py::none(), py::arg("root_q_end") = py::none())
        .def("reset_envs",
             [](RopeBatch& b, py::array_t<int, py::array::c_style | py::array::forcecast> ids) {
                 if (ids.ndim() != 1) throw py::value_error("ids must be 1-D");
                 if (ids.shape(0) > b.R) throw py::value_error("ids longer than num_envs");
                 std::vector<int> v(ids.data(), ids.data() + ids.shape(0));
                 for (int i : v)
                     if (i < 0 || i >= b.R) throw py::value_error("env id out of range");
                 py::gil_scoped_release rel;
                 ok(rs_batch_reset_ropes(b.h, v.data(), (int)v.size()));
             },
             py::arg("ids"))
        .def("gather", [](RopeBatch& b) {
            py::gil_scoped_release rel;
            ok(rs_batch_gather(b.h));
        })
        .def("positions", [](RopeBatch& b) {
            float* p; ok(rs_batch_views(b.h, &p, nullptr, nullptr));
            return CudaView{(uintptr_t)p, b.vshape(3)};
        }, py::keep_alive<0, 1>())
        .def("velocities", [](RopeBatch& b) {
            float* p; ok(rs_batch_views(b.h, nullptr, &p, nullptr));
            return CudaView{(uintptr_t)p, b.vshape(3)};
        }, py::keep_alive<0, 1>())
        .def("quaternions", [](RopeBatch& b) {
            float* p; ok(rs_batch_views(b.h, nullptr, nullptr, &p));
            return CudaView{(uintptr_t)p, b.vshape(4)};
        }, py::keep_alive<0, 1>())
        .def_property("drag", [](RopeBatch& b) { return b.get(RS_P_DRAG); }, [](RopeBatch& b, float v) { b.set(RS_P_DRAG, v); })
        .def_property("drag_quad", [](RopeBatch& b) { return b.get(RS_P_DRAG_QUAD); },
                      [](RopeBatch& b, float v) { b.set(RS_P_DRAG_QUAD, v); })
        .def_property("drag_quad_t", [](RopeBatch& b) { return b.get(RS_P_DRAG_QUAD_T); },
                      [](RopeBatch& b, float v) { b.set(RS_P_DRAG_QUAD_T, v); })
        .def_property("damping", [](RopeBatch& b) { return b.get(RS_P_DAMPING); },
                      [](RopeBatch& b, float v) { b.set(RS_P_DAMPING, v); })
        .def_property("num_itr", [](RopeBatch& b) { int v; ok(rs_batch_get_num_itr(b.h, &v)); return v; },
                      [](RopeBatch& b, int v) {
                          if (v < 1) throw py::value_error("num_itr must be >= 1");
                          ok(rs_batch_set_num_itr(b.h, v));
                      })
        .def_property("accel_ratio", [](RopeBatch& b) { return b.get(RS_P_ACCEL); },
                      [](RopeBatch& b, float v) { b.set(RS_P_ACCEL, v); })
        .def_static("from_positions",
             [](farray pos, float density, float k_stretch, float k_bend, float max_h, int num_itr, bool fix_root_orientation,
                py::object pinned, bool straight_rest, bool deterministic) {
                 (void)deterministic;
                 if (pos.ndim() != 3 || pos.shape(2) != 3 || pos.shape(1) < 3)
                     throw py::value_error("positions must be [num_envs, V>=3, 3]");
                 const int N = (int)pos.shape(0), V = (int)pos.shape(1);
                 if (!(density > 0) || !(k_stretch > 0) || !(k_bend > 0) || !(max_h > 0) || num_itr < 1)
                     throw py::value_error("density, k_stretch, k_bend, max_h > 0 and num_itr >= 1 required");
                 std::vector<uint8_t> pin((size_t)N * V, 0);
                 if (pinned.is_none()) {
                     for (int e = 0; e < N; e++) pin[(size_t)e * V] = 1;
                 } else {
                     auto pm = pinned.cast<py::array_t<bool, py::array::c_style | py::array::forcecast>>();
                     const bool per_env = pm.ndim() == 2;
                     if (!((pm.ndim() == 1 && pm.shape(0) == V) || (per_env && pm.shape(0) == N && pm.shape(1) == V)))
                         throw py::value_error("pinned must be [V] or [num_envs, V] booleans");
                     for (int e = 0; e < N; e++)
                         for (int v = 0; v < V; v++) pin[(size_t)e * V + v] = pm.data()[per_env ? (size_t)e * V + v : (size_t)v];
                 }
                 if (fix_root_orientation)
                     for (int e = 0; e < N; e++)
                         if (!pin[(size_t)e * V]) throw py::value_error("fix_root_orientation=True needs every root pinned");
                 const float* p = pos.data();
                 float minSeg = 1e30f;
                 for (int e = 0; e < N; e++)
                     for (int v = 0; v < V; v++) {
                         const float* a = p + ((size_t)e * V + v) * 3;
                         if (!std::isfinite(a[0]) || !std::isfinite(a[1]) || !std::isfinite(a[2]))
                             throw py::value_error("positions must be finite");
                         if (v + 1 < V) {
                             const float dx = a[3] - a[0], dy = a[4] - a[1], dz = a[5] - a[2];
                             const float l = std::sqrt(dx * dx + dy * dy + dz * dz);
                             if (!(l > 0)) throw py::value_error("consecutive vertices must not coincide");
                             minSeg = std::min(minSeg, l);
                         }
                     }
                 return make_batch(N, std::vector<int>(N, V), p, pin.data(), density, k_stretch, k_bend, max_h, num_itr,
                                   fix_root_orientation, straight_rest, minSeg);
             },
             py::arg("positions"), py::arg("density"), py::arg("k_stretch"), py::arg("k_bend"), py::arg("max_h"),
             py::arg("num_itr"), py::arg("fix_root_orientation") = false, py::arg("pinned") = py::none(),
             py::arg("straight_rest") = false, py::arg("deterministic") = false)
        .def_static("from_ropes",
             [](py::list ropes, float density, float k_stretch, float k_bend, float max_h, int num_itr, bool fix_root_orientation,
                py::object pinned, bool straight_rest) {
                 // uneven ropes (new surface): a list of [V_r, 3] arrays, optional list of [V_r] pin masks
                 const int N = (int)py::len(ropes);
                 if (N < 1) throw py::value_error("ropes must be a non-empty list of [V_r >= 3, 3] arrays");
                 std::vector<int> verts;
                 std::vector<float> pos;
                 std::vector<uint8_t> pin;
                 float minSeg = 1e30f;
                 for (int r = 0; r < N; r++) {
                     farray a = ropes[r].cast<farray>();
                     if (a.ndim() != 2 || a.shape(1) != 3 || a.shape(0) < 3)
                         throw py::value_error("every rope must be a [V_r >= 3, 3] array");
                     const int V = (int)a.shape(0);
                     verts.push_back(V);
                     for (int i = 0; i < 3 * V; i++) {
                         if (!std::isfinite(a.data()[i])) throw py::value_error("positions must be finite");
                         pos.push_back(a.data()[i]);
                     }
                     for (int v = 0; v + 1 < V; v++) {
                         const float* q = a.data() + 3 * v;
                         const float l = std::sqrt((q[3] - q[0]) * (q[3] - q[0]) + (q[4] - q[1]) * (q[4] - q[1]) + (q[5] - q[2]) * (q[5] - q[2]));
                         if (!(l > 0)) throw py::value_error("consecutive vertices must not coincide");
                         minSeg = std::min(minSeg, l);
                     }
                     if (pinned.is_none()) {
                         for (int v = 0; v < V; v++) pin.push_back(v == 0 ? 1 : 0);
                     } else {
                         auto pm = pinned.cast<py::list>()[r].cast<py::array_t<bool, py::array::c_style | py::array::forcecast>>();
                         if (pm.ndim() != 1 || pm.shape(0) != V) throw py::value_error("pinned[r] must be [V_r] booleans");
                         for (int v = 0; v < V; v++) pin.push_back(pm.data()[v] ? 1 : 0);
                     }
                     if (fix_root_orientation && !pin[pin.size() - V])
                         throw py::value_error("fix_root_orientation=True needs every root pinned");
                 }
                 if (!(density > 0) || !(k_stretch > 0) || !(k_bend > 0) || !(max_h > 0) || num_itr < 1)
                     throw py::value_error("density, k_stretch, k_bend, max_h > 0 and num_itr >= 1 required");
                 return make_batch(N, verts, pos.data(), pin.data(), density, k_stretch, k_bend, max_h, num_itr,
                                   fix_root_orientation, straight_rest, minSeg);
             },
             py::arg("ropes"), py::arg("density"), py::arg("k_stretch"), py::arg("k_bend"), py::arg("max_h"),
             py::arg("num_itr"), py::arg("fix_root_orientation") = false, py::arg("pinned") = py::none(),
             py::arg("straight_rest") = false)
        .def("set_rope_contact",
             [](RopeBatch& b, bool enabled, float radius, float barrier, float k_collision, float mu, float k_friction,
                float detection_scaler, int group_ropes) {
                 if (enabled && (!(radius > 0) || !(barrier > 0) || !(k_collision > 0) || !(mu >= 0) || !(k_friction >= 0) ||
                                 !(detection_scaler > 1) || group_ropes < 1))
                     throw py::value_error("rope contact needs radius, barrier, k_collision > 0, mu, k_friction >= 0, "
                                           "detection_scaler > 1, group_ropes >= 1");
                 ok(rs_batch_set_rope_contact(b.h, enabled ? 1 : 0, radius, barrier, k_collision, mu, k_friction,
                                              detection_scaler, group_ropes));
             },
             py::arg("enabled"), py::arg("radius") = 0.f, py::arg("barrier") = 0.f, py::arg("k_collision") = 0.f,
             py::arg("mu") = 0.f, py::arg("k_friction") = 0.f, py::arg("detection_scaler") = 1.2f, py::arg("group_ropes") = 1)
        .def("step_free",
             [](RopeBatch& b, float dt, int substeps) {
                 if (!(dt > 0) || substeps < 1) throw py::value_error("dt > 0 and substeps >= 1 required");
                 b.stepped = true;
                 py::gil_scoped_release rel;
                 ok(rs_batch_step_free(b.h, dt, substeps));
             },
             py::arg("dt"), py::arg("substeps"))
        // ---- differentiable frames (no counterpart in the reference; see ropesim.grad)
        .def("set_state",
             [](RopeBatch& b, py::object pos, py::object vel, py::object lvel, py::object q) {
                 const uintptr_t p = parse_vertex_array(pos, b.n, b.R, b.V, 3, "pos");
                 const uintptr_t v = parse_vertex_array(vel, b.n, b.R, b.V, 3, "vel");
                 const uintptr_t l = parse_vertex_array(lvel, b.n, b.R, b.V, 3, "lvel");
                 const uintptr_t qq = parse_vertex_array(q, b.n, b.R, b.V, 4, "q");
                 py::gil_scoped_release rel;
                 ok(rs_batch_set_state(b.h, (const float*)p, (const float*)v, (const float*)l, (const float*)qq, 1));
             },
             py::arg("pos"), py::arg("vel"), py::arg("lvel"), py::arg("q"))
        .def("get_state",
             [](RopeBatch& b, py::object pos, py::object vel, py::object lvel, py::object q) {
                 const uintptr_t p = parse_vertex_array(pos, b.n, b.R, b.V, 3, "pos");
                 const uintptr_t v = parse_vertex_array(vel, b.n, b.R, b.V, 3, "vel");
                 const uintptr_t l = parse_vertex_array(lvel, b.n, b.R, b.V, 3, "lvel");
                 const uintptr_t qq = parse_vertex_array(q, b.n, b.R, b.V, 4, "q");
                 py::gil_scoped_release rel;
                 ok(rs_batch_get_state(b.h, (float*)p, (float*)v, (float*)l, (float*)qq, 1));
             },
             py::arg("pos"), py::arg("vel"), py::arg("lvel"), py::arg("q"))
        .def("set_parameters",
             [](RopeBatch& b, py::object ea, py::object ei, py::object mass) {
                 const uintptr_t a = parse_vertex_array(ea, b.n, b.R, b.V, 0, "ea");
                 const uintptr_t e = parse_vertex_array(ei, b.n, b.R, b.V, 0, "ei");
                 const uintptr_t m = parse_vertex_array(mass, b.n, b.R, b.V, 0, "mass");
                 py::gil_scoped_release rel;
                 ok(rs_batch_set_parameters(b.h, (const float*)a, (const float*)e, (const float*)m, 1));
             },
             py::arg("ea"), py::arg("ei"), py::arg("mass"))
        .def("get_parameters",
             [](RopeBatch& b, py::object ea, py::object ei, py::object mass) {
                 const uintptr_t a = parse_vertex_array(ea, b.n, b.R, b.V, 0, "ea");
                 const uintptr_t e = parse_vertex_array(ei, b.n, b.R, b.V, 0, "ei");
                 const uintptr_t m = parse_vertex_array(mass, b.n, b.R, b.V, 0, "mass");
                 py::gil_scoped_release rel;
                 ok(rs_batch_get_parameters(b.h, (float*)a, (float*)e, (float*)m, 1));
             },
             py::arg("ea"), py::arg("ei"), py::arg("mass"))
        .def_property_readonly("current_h",
                               [](RopeBatch& b) {
                                   float v = 0.f;
                                   ok(rs_batch_get_param(b.h, RS_P_H, &v));
                                   return v;
                               })
        // Low-level reverse of one frame, queued on the handle's stream: 28 device pointers in
        // rs_backward_io order (0 = NULL); ropesim.grad validates the tensors behind them.
        .def("_backward",
             [](RopeBatch& b, std::vector<uintptr_t> ptrs, float dt, int substeps, float last_h) {
                 if (ptrs.size() != 28) throw py::value_error("_backward expects 28 pointers");
                 rs_backward_io io;
                 const float** c = reinterpret_cast<const float**>(&io);
                 for (int i = 0; i < 28; i++) c[i] = reinterpret_cast<const float*>(ptrs[i]);
                 py::gil_scoped_release rel;
                 ok(rs_batch_backward_async(b.h, &io, dt, substeps, last_h));
             },
             py::arg("ptrs"), py::arg("dt"), py::arg("substeps"), py::arg("last_h"))
        // One differentiable frame in one call, queued on the handle's stream: 16 device pointers in
        // rs_frame_io order; returns the frame's lastH.
        .def("_frame_forward",
             [](RopeBatch& b, std::vector<uintptr_t> ptrs, float dt, int substeps) {
                 if (ptrs.size() != 16) throw py::value_error("_frame_forward expects 16 pointers");
                 rs_frame_io io;
                 const float** c = reinterpret_cast<const float**>(&io);
                 for (int i = 0; i < 16; i++) c[i] = reinterpret_cast<const float*>(ptrs[i]);
                 float lh = 0.f;
                 b.stepped = true;
                 {
                     py::gil_scoped_release rel;
                     ok(rs_batch_frame_forward(b.h, &io, dt, substeps, &lh));
                 }
                 return lh;
             },
             py::arg("ptrs"), py::arg("dt"), py::arg("substeps"))
        // Program step recording the substep tape into a caller buffer of 16 * substeps * n floats.
        .def("_step_taped",
             [](RopeBatch& b, py::object root_pos, py::object root_vel, py::object root_pos_end, float dt, int substeps,
                uintptr_t tape) {
                 if (!(dt > 0) || substeps < 1) throw py::value_error("dt > 0 and substeps >= 1 required");
                 if (!b.rootsPinned) throw py::value_error("the program step drives every rope's root");
                 const uintptr_t p = parse_cai(root_pos, {b.R, 3}, "root_pos");
                 const uintptr_t v = parse_cai(root_vel, {b.R, 3}, "root_vel");
                 const uintptr_t p1 = parse_cai(root_pos_end, {b.R, 3}, "root_pos_end");
                 b.stepped = true;
                 py::gil_scoped_release rel;
                 ok(rs_batch_step_program_taped(b.h, (const float*)p, (const float*)v, (const float*)p1, nullptr, nullptr,
                                                dt, substeps, (float*)tape));
             },
             py::arg("root_pos"), py::arg("root_vel"), py::arg("root_pos_end"), py::arg("dt"), py::arg("substeps"),
             py::arg("tape"))
        .def("set_velocities",
             [](RopeBatch& b, farray v) {
                 if (b.V > 0) {
                     if (v.ndim() != 3 || v.shape(0) != b.R || v.shape(1) != b.V || v.shape(2) != 3)
                         throw py::value_error("expected [num_envs, V, 3]");
                 } else if (v.ndim() != 2 || v.shape(0) != b.n || v.shape(1) != 3) {
                     throw py::value_error("expected [total_verts, 3]");
                 }
                 ok(rs_batch_set_velocities(b.h, v.data()));
             },
             py::arg("velocities"))
        .def("set_planes", &RopeBatch::set_planes, py::arg("planes"), py::arg("radius") = 0.f, py::arg("mu_s") = 0.5f,
             py::arg("mu_k") = py::none(), py::arg("v_slip") = 1e-3f, py::arg("kappa") = 2.f)
        .def("set_contact", &RopeBatch::set_contact, py::arg("radius"), py::arg("mu_s") = 0.5f, py::arg("mu_k") = py::none(),
             py::arg("v_slip") = 1e-3f, py::arg("kappa") = 2.f)
        .def("add_mesh",
             [](RopeBatch& b, farray values, farray origin, float spacing, farray pos, farray quat, py::object mu_s,
                py::object mu_k) { return b.add_mesh(values, origin, spacing, pos, quat, mu_s, mu_k, b.R); },
             py::arg("values"), py::arg("origin"), py::arg("spacing"),
             py::arg("pos") = farray(py::cast(std::vector<float>{0, 0, 0})),
             py::arg("quat") = farray(py::cast(std::vector<float>{0, 0, 0, 1})), py::arg("mu_s") = py::none(),
             py::arg("mu_k") = py::none())
        .def("set_mesh_friction", &RopeBatch::set_mesh_friction, py::arg("index"), py::arg("mu_s"), py::arg("mu_k") = py::none())
        .def("set_mesh_poses",
             [](RopeBatch& b, int index, py::object pos, py::object quat, py::object teleport) {
                 const bool dp = py::hasattr(pos, "__cuda_array_interface__"), dq = py::hasattr(quat, "__cuda_array_interface__");
                 if (dp != dq) throw py::value_error("set_mesh_poses: pos and quat must both be host arrays or both CUDA arrays");
                 const Tele t = parse_teleport(teleport, b.R, "set_mesh_poses");
                 if (dp) {
                     const uintptr_t p = parse_cai(pos, {b.R, 3}, "pos"), q = parse_cai(quat, {b.R, 4}, "quat");
                     if (t.device) {
                         ok(rs_batch_set_mesh_poses(b.h, index, (const float*)p, (const float*)q, b.R, t.ptr, 0, 1));
                     } else if (!t.all && t.ptr) {  // host flags with device poses: the library stages them
                         ok(rs_batch_set_mesh_poses(b.h, index, (const float*)p, (const float*)q, b.R, t.ptr, 0, 3));
                     } else {
                         ok(rs_batch_set_mesh_poses(b.h, index, (const float*)p, (const float*)q, b.R, nullptr, t.all ? 1 : 0, 1));
                     }
                     return;
                 }
                 if (t.device) throw py::value_error("set_mesh_poses: host poses need teleport as a bool or a host bool array");
                 farray hp = farray::ensure(pos), hq = farray::ensure(quat);
                 if (!hp || !hq) throw py::value_error("set_mesh_poses: pos/quat must be arrays");
                 const int rows = parse_poses(hp, hq, b.R, "set_mesh_poses");
                 ok(rs_batch_set_mesh_poses(b.h, index, hp.data(), hq.data(), rows, t.all ? nullptr : t.ptr, t.all ? 1 : 0, 0));
             },
             py::arg("index"), py::arg("pos"), py::arg("quat"), py::arg("teleport") = false)
        .def("set_mesh_poses_all",
             [](RopeBatch& b, py::object pos, py::object quat, py::object teleport) {
                 const int N = b.R, M = b.meshes();
                 const Tele t = parse_teleport(teleport, N, "set_mesh_poses_all");
                 const bool dp = py::hasattr(pos, "__cuda_array_interface__"), dq = py::hasattr(quat, "__cuda_array_interface__");
                 if (dp != dq) throw py::value_error("set_mesh_poses_all: pos and quat must both be host arrays or both CUDA arrays");
                 if (dp) {
                     const uintptr_t p = parse_cai(pos, {N, M, 3}, "pos"), q = parse_cai(quat, {N, M, 4}, "quat");
                     const bool host_flags = !t.device && !t.all && t.ptr;  // staged by the library
                     ok(rs_batch_set_mesh_poses(b.h, -1, (const float*)p, (const float*)q, N * M, t.all ? nullptr : t.ptr,
                                                t.all ? 1 : 0, host_flags ? 3 : 1));
                     return;
                 }
                 if (t.device) throw py::value_error("set_mesh_poses_all: host poses need teleport as a bool or a host bool array");
                 farray hp = farray::ensure(pos), hq = farray::ensure(quat);
                 if (!hp || !hq || hp.ndim() != 3 || hq.ndim() != 3 || hp.shape(0) != N || hq.shape(0) != N || hp.shape(1) != M ||
                     hq.shape(1) != M || hp.shape(2) != 3 || hq.shape(2) != 4)
                     throw py::value_error("set_mesh_poses_all: pos must be [num_envs, num_meshes, 3] and quat [num_envs, num_meshes, 4]");
                 validate_rows(hp.data(), hq.data(), N * M, "set_mesh_poses_all");
                 ok(rs_batch_set_mesh_poses(b.h, -1, hp.data(), hq.data(), N * M, t.all ? nullptr : t.ptr, t.all ? 1 : 0, 0));
             },
             py::arg("pos"), py::arg("quat"), py::arg("teleport") = false)
        .def("clear_meshes", [](RopeBatch& b) { ok(rs_batch_clear_meshes(b.h)); })
        .def("enable_contact_forces", [](RopeBatch& b, bool on) { ok(rs_batch_enable_contact_forces(b.h, on ? 1 : 0)); },
             py::arg("on") = true)
        .def("contact_forces_view", [](RopeBatch& b) {
            float *f = nullptr, *w = nullptr;
            ok(rs_batch_contact_views(b.h, &f, &w));
            return CudaView{(uintptr_t)f, b.vshape(3)};
        }, py::keep_alive<0, 1>())
        .def("mesh_wrenches_view", [](RopeBatch& b) {
            float *f = nullptr, *w = nullptr;
            ok(rs_batch_contact_views(b.h, &f, &w));
            return CudaView{(uintptr_t)w, {b.R, 64, 6}};
        }, py::keep_alive<0, 1>())
        .def("contact_forces", [](RopeBatch& b) {
            py::array_t<float> out(b.vshape(3));
            ok(rs_batch_contact_forces(b.h, out.mutable_data()));
            return out;
        })
        .def("mesh_wrenches", [](RopeBatch& b) {
            py::array_t<float> out({(py::ssize_t)b.R, (py::ssize_t)b.meshes(), (py::ssize_t)6});
            ok(rs_batch_mesh_wrenches(b.h, out.mutable_data()));
            return out;
        })
        .def("set_gravity", [](RopeBatch& b, farray g) { ok(rs_batch_set_gravity(b.h, vec3(g, "gravity").data())); }, py::arg("gravity"))
        .def("inv_masses", [](RopeBatch& b) {
            py::array_t<float> a(b.V > 0 ? std::vector<py::ssize_t>{b.R, b.V} : std::vector<py::ssize_t>{b.n});
            ok(rs_batch_inv_masses(b.h, a.mutable_data()));
            return a;
        })
        .def("set_masses",
             [](RopeBatch& b, farray m) {
                 if (b.stepped) throw py::value_error("set_masses is only legal before the first step");
                 auto v = b.per_vertex(m, 0, "expected [V] or [num_envs, V] node masses (kg)");
                 ok(rs_batch_set_masses(b.h, v.data()));
             },
             py::arg("masses"))
        .def("set_stretch_stiffnesses",
             [](RopeBatch& b, farray ea) {
                 if (b.stepped) throw py::value_error("set_stretch_stiffnesses is only legal before the first step");
                 auto v = b.per_vertex(ea, 1, "expected [V-1] or [num_envs, V-1] EA values");
                 ok(rs_batch_set_stretch_stiffnesses(b.h, v.data()));
             },
             py::arg("ea"))
        .def("set_bend_stiffnesses",
             [](RopeBatch& b, farray ei) {
                 if (b.stepped) throw py::value_error("set_bend_stiffnesses is only legal before the first step");
                 auto v = b.per_vertex(ei, 1, "expected [V-1] or [num_envs, V-1] EI values");
                 ok(rs_batch_set_bend_stiffnesses(b.h, v.data()));
             },
             py::arg("ei"))
        .def("set_block", [](RopeBatch& b, int block) { ok(rs_batch_set_block(b.h, block)); }, py::arg("block"))
        .def("layout", [](RopeBatch& b) {
            int blk = 0, nb = 0;
            ok(rs_batch_layout(b.h, &blk, &nb));
            return py::make_tuple(blk, nb);
        })
        .def("set_sync", [](RopeBatch& b, bool every_frame) { ok(rs_batch_set_sync(b.h, every_frame ? 1 : 0)); })
        .def("set_autotune", [](RopeBatch& b, bool on) { ok(rs_batch_set_autotune(b.h, on ? 1 : 0)); })
        .def("set_culling", [](RopeBatch& b, bool on) { ok(rs_batch_set_culling(b.h, on ? 1 : 0)); }, py::arg("on"))
        .def("set_work_queue", [](RopeBatch& b, bool on) { ok(rs_batch_set_work_queue(b.h, on ? 1 : 0)); }, py::arg("on"))
        .def("set_engine", [](RopeBatch& b, const std::string& e) {
            if (e != "persistent" && e != "plain") throw py::value_error("engine must be 'persistent' or 'plain'");
            ok(rs_batch_set_engine(b.h, e == "plain" ? 1 : 0));
        }, py::arg("engine"))
        .def("set_timing", [](RopeBatch& b, bool on) { ok(rs_batch_set_timing(b.h, on ? 1 : 0)); })
        .def("last_frame_ms", [](RopeBatch& b) { double ms = 0; ok(rs_batch_last_frame_ms(b.h, &ms)); return ms; })
        .def("stream_ptr", [](RopeBatch& b) { void* s = nullptr; ok(rs_batch_stream(b.h, &s)); return (uintptr_t)s; })
        .def_property_readonly("time", [](RopeBatch& b) { return b.get(RS_P_TIME); })
        .def_property_readonly("last_error", [](RopeBatch& b) { int e; ok(rs_batch_status(b.h, &e, nullptr, nullptr)); return e; })
        .def_property_readonly("last_warning", [](RopeBatch& b) { int w; ok(rs_batch_status(b.h, nullptr, &w, nullptr)); return w; })
        .def_property_readonly("nonfinite", [](RopeBatch& b) { int f; ok(rs_batch_status(b.h, nullptr, nullptr, &f)); return f; })
        .def("bounds_check", [](RopeBatch& b) {
            int code = 0, checked = 0;
            ok(rs_batch_bounds_check(b.h, &code, &checked));
            return py::make_tuple(code, (bool)checked);
        })
        .def_property_readonly("num_envs", [](RopeBatch& b) { return b.R; })
        .def_property_readonly("verts_per_rope", [](RopeBatch& b) { return b.V; })
        .def_property_readonly("rope_verts", [](RopeBatch& b) { return b.verts; })
        .def_property_readonly("num_verts", [](RopeBatch& b) { return b.n; })
        .def_property_readonly("fixed_root_orientation", [](RopeBatch& b) { return b.fixRoot; });
}
