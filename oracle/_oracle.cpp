// _oracle.cpp -- TEST INFRASTRUCTURE ONLY: pybind11 binding of the CPU restatement in
// rs_oracle.hpp (Sim64 = double, Sim32 = float). Arrays in and out are numpy; inputs are
// validated by the Python wrapper (ropesim_oracle.py), which mirrors the ropesim API.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <chrono>
#include <thread>

#include "rs_adjoint.hpp"
#include "rs_opcount.hpp"
#include "rs_oracle.hpp"
#include "rs_sdfbake_oracle.hpp"

namespace py = pybind11;
using f32a = py::array_t<float, py::array::c_style | py::array::forcecast>;
using i32a = py::array_t<int, py::array::c_style | py::array::forcecast>;
using u8a = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>;
using f64a = py::array_t<double, py::array::c_style | py::array::forcecast>;

template <class T>
static void v3_in(std::vector<rso::V3<T>>& v, const f64a& a) {
    const double* p = a.data();
    for (size_t i = 0; i < v.size(); i++) v[i] = rso::V3<T>(T(p[3 * i]), T(p[3 * i + 1]), T(p[3 * i + 2]));
}
template <class T>
static void q4_in(std::vector<rso::Q4<T>>& v, const f64a& a) {
    const double* p = a.data();
    for (size_t i = 0; i < v.size(); i++) v[i] = rso::Q4<T>(T(p[4 * i]), T(p[4 * i + 1]), T(p[4 * i + 2]), T(p[4 * i + 3]));
}

template <class T>
static py::array_t<double> v3_out(const std::vector<rso::V3<T>>& v) {
    py::array_t<double> a({(py::ssize_t)v.size(), (py::ssize_t)3});
    auto m = a.mutable_unchecked<2>();
    for (size_t i = 0; i < v.size(); i++) { m(i, 0) = (double)v[i].x; m(i, 1) = (double)v[i].y; m(i, 2) = (double)v[i].z; }
    return a;
}
template <class T>
static py::array_t<double> q4_out(const std::vector<rso::Q4<T>>& v) {
    py::array_t<double> a({(py::ssize_t)v.size(), (py::ssize_t)4});
    auto m = a.mutable_unchecked<2>();
    for (size_t i = 0; i < v.size(); i++) { m(i, 0) = (double)v[i].x; m(i, 1) = (double)v[i].y; m(i, 2) = (double)v[i].z; m(i, 3) = (double)v[i].w; }
    return a;
}
template <class T>
static py::array_t<double> s_out(const std::vector<T>& v) {
    py::array_t<double> a((py::ssize_t)v.size());
    auto m = a.mutable_unchecked<1>();
    for (size_t i = 0; i < v.size(); i++) m(i) = (double)v[i];
    return a;
}
static const float* opt_ptr(const py::object& o, f32a& keep) {
    if (o.is_none()) return nullptr;
    keep = f32a::ensure(o);
    return keep.data();
}

template <class T>
static py::class_<rso::Sim<T>> bind_sim(py::module_& m, const char* name) {
    using S = rso::Sim<T>;
    py::class_<S> cls(m, name);
    cls
        .def(py::init([](f32a positions, i32a starts, u8a pinned, float density, float ks, float kb, float max_h, int num_itr,
                         bool fix_root, bool straight_rest, bool per_rope_env, float dead_r, float dead_b) {
                 return new S(positions.data(), starts.data(), (int)starts.shape(0) - 1, pinned.data(), density, ks, kb, max_h,
                              num_itr, fix_root, straight_rest, per_rope_env, dead_r, dead_b);
             }),
             py::arg("positions"), py::arg("starts"), py::arg("pinned"), py::arg("density"), py::arg("k_stretch"),
             py::arg("k_bend"), py::arg("max_h"), py::arg("num_itr"), py::arg("fix_root_orientation"),
             py::arg("straight_rest"), py::arg("per_rope_env"), py::arg("dead_radius"), py::arg("dead_barrier"))
        .def_readonly("n", &S::n)
        .def_readonly("num_ropes", &S::R)
        .def_property("gravity", [](S& s) { return std::vector<double>{(double)s.gravity.x, (double)s.gravity.y, (double)s.gravity.z}; },
                      [](S& s, std::vector<double> g) { s.gravity = rso::V3<T>(T((float)g[0]), T((float)g[1]), T((float)g[2])); })
        .def_property("drag", [](S& s) { return (double)s.drag; }, [](S& s, float v) { s.drag = T(v); })
        .def_property("drag_quad", [](S& s) { return (double)s.dragQuad; }, [](S& s, float v) { s.dragQuad = T(v); })
        .def_property("drag_quad_t", [](S& s) { return (double)s.dragQuadT; }, [](S& s, float v) { s.dragQuadT = T(v); })
        .def_property("damping", [](S& s) { return (double)s.damping; }, [](S& s, float v) { s.damping = T(v); })
        .def_property("inplace_frames", [](S& s) { return s.inplaceFrames; }, [](S& s, bool v) { s.inplaceFrames = v; })
        .def_property("accel_ratio", [](S& s) { return (double)s.accel; }, [](S& s, float v) { s.accel = T(v); })
        .def_property("num_itr", [](S& s) { return s.numItr; }, [](S& s, int v) { s.numItr = v; })
        .def_property("max_h", [](S& s) { return s.maxH; }, [](S& s, float v) { s.maxH = v; })
        .def_property_readonly("time", [](S& s) { return (double)s.time; })
        .def_property_readonly("h", [](S& s) { return (double)s.h; })
        .def_property_readonly("last_error", [](S& s) { return s.lastError; })
        .def_property_readonly("last_warning", [](S& s) { return s.lastWarning; })
        .def_property_readonly("min_seg_len", [](S& s) { return (double)s.minSegLen; })
        .def("set_contact", [](S& s, float r, float ms, float mk, float vs, float ka) { s.set_contact(T(r), T(ms), T(mk), T(vs), T(ka)); })
        .def("set_planes", [](S& s, f32a rows) { s.set_planes((int)rows.shape(0), rows.data()); })
        .def("set_rope_contact", [](S& s, bool on, float r, float b, float kc, float mu, float kf, float sc, int g) {
            s.set_rope_contact(on, T(r), T(b), T(kc), T(mu), T(kf), T(sc), g);
        })
        .def("add_mesh", [](S& s, f32a values, f32a origin, float spacing, float ms, float mk, f32a p, f32a q, int rows) {
            return s.add_mesh(values.data(), (int)values.shape(0), (int)values.shape(1), (int)values.shape(2), origin.data(),
                              spacing, ms, mk, p.data(), q.data(), rows);
        })
        .def("set_mesh_friction", [](S& s, int i, float ms, float mk) { s.set_mesh_friction(i, T(ms), T(mk)); })
        .def("set_targets", [](S& s, int index, f32a p, f32a q, int rows, py::object tele, bool tele_all) {
            u8a tk;
            const uint8_t* tp = nullptr;
            if (!tele.is_none()) { tk = u8a::ensure(tele); tp = tk.data(); }
            s.set_targets(index, p.data(), q.data(), rows, tp, tele_all);
        })
        .def("clear_meshes", &S::clear_meshes)
        .def("enable_forces", &S::enable_forces)
        .def_property_readonly("num_meshes", [](S& s) { return (int)s.grids.size(); })
        .def("set_vertex_ea", [](S& s, int i, float v) { s.set_vertex_ea(i, T(v)); })
        .def("set_vertex_ei", [](S& s, int i, float v) { s.set_vertex_ei(i, T(v)); })
        .def("set_vertex_mass", [](S& s, int i, float v) { s.set_vertex_mass(i, T(v)); })
        .def("set_root", [](S& s, int r, f32a p, f32a v, py::object q) {
            const int root = s.start[r];
            s.pos[root] = rso::V3<T>(T(p.data()[0]), T(p.data()[1]), T(p.data()[2]));
            s.vel[root] = rso::V3<T>(T(v.data()[0]), T(v.data()[1]), T(v.data()[2]));
            if (!q.is_none()) {
                f32a qa = f32a::ensure(q);  // already unit (normalized by the caller in float)
                s.q[root] = rso::Q4<T>(T(qa.data()[0]), T(qa.data()[1]), T(qa.data()[2]), T(qa.data()[3]));
            }
        })
        .def("set_velocities", [](S& s, f32a v) {
            for (int i = 0; i < s.n; i++) s.vel[i] = rso::V3<T>(T(v.data()[3 * i]), T(v.data()[3 * i + 1]), T(v.data()[3 * i + 2]));
        })
        .def("unpin_root", [](S& s) { s.invMass[0] = T(2) * s.invMass[1]; s.vel[0] = rso::V3<T>(); })
        .def("advance", &S::advance, py::call_guard<py::gil_scoped_release>())
        .def("step_legacy", [](S& s, f32a p, f32a v, py::object q, float dt, int S_) {
            f32a kq;
            const float* qp = opt_ptr(q, kq);
            py::gil_scoped_release rel;
            s.step_legacy(p.data(), v.data(), qp, dt, S_);
        })
        .def("step_program", [](S& s, f32a p0, f32a v0, f32a p1, py::object q0, py::object q1, float dt, int S_) {
            f32a k0, k1;
            const float* a = opt_ptr(q0, k0);
            const float* b = opt_ptr(q1, k1);
            py::gil_scoped_release rel;
            s.step_program(p0.data(), v0.data(), p1.data(), a, b, dt, S_);
        })
        .def("step_free", &S::step_free, py::call_guard<py::gil_scoped_release>())
        .def("reset_ropes", [](S& s, i32a ids) { s.reset_ropes(ids.data(), (int)ids.shape(0)); })
        .def("reset_all", &S::reset_all)
        .def("positions", [](S& s) { return v3_out(s.pos); })
        .def("velocities", [](S& s) { return v3_out(s.vel); })
        .def("quaternions", [](S& s) { return q4_out(s.q); })
        .def("rest_rotations", [](S& s) { return q4_out(s.qRest); })
        .def("inv_masses", [](S& s) { return s_out(s.invMass); })
        .def("rest_lengths", [](S& s) { return s_out(s.lRest); })
        .def("k_stretch", [](S& s) { return s_out(s.kStretch); })
        .def("flags", [](S& s) { return std::vector<uint32_t>(s.flags.begin(), s.flags.end()); })
        .def("last_velocities", [](S& s) { return v3_out(s.lastVel); })
        .def_property_readonly("last_h", [](S& s) { return (double)s.lastH; })
        // Full dynamic state (pos, vel, lastVel, q, h, lastH) in double, for the adjoint checks.
        .def("get_state", [](S& s) {
            return py::make_tuple(v3_out(s.pos), v3_out(s.vel), v3_out(s.lastVel), q4_out(s.q), (double)s.h, (double)s.lastH);
        })
        .def("set_state", [](S& s, f64a pos, f64a vel, f64a lv, f64a q, double h, double lastH) {
            v3_in(s.pos, pos); v3_in(s.vel, vel); v3_in(s.lastVel, lv); q4_in(s.q, q);
            s.h = T(h); s.lastH = T(lastH);
        })
        // Differentiated parameters: kStretch (EA l), |qRest| (4 EI / l), invMass.
        .def("get_params", [](S& s) {
            std::vector<T> rho(s.n);
            for (int i = 0; i < s.n; i++) rho[i] = rso::len4(s.qRest[i]);
            return py::make_tuple(s_out(s.kStretch), s_out(rho), s_out(s.invMass));
        })
        .def("set_params", [](S& s, f64a ks, f64a rho, f64a w) {
            for (int i = 0; i < s.n; i++) {
                s.kStretch[i] = T(ks.data()[i]);
                const T l = rso::len4(s.qRest[i]);
                if (l > 0) s.qRest[i] = s.qRest[i] * (T(rho.data()[i]) / l);
                s.invMass[i] = T(w.data()[i]);
            }
        })
        .def("step_program_rows", [](S& s, f64a prog, float dt, int S_) {
            std::vector<T> p(prog.data(), prog.data() + prog.size());
            py::gil_scoped_release rel;
            s.step_program_rows(p.data(), dt, S_);
        })
        .def("rope_contact_counts", [](S& s) {  // (active rope-rope terms, limited steps) since the last call
            const auto r = py::make_tuple(s.nCollisionTerms, s.nLimitedSteps);
            s.nCollisionTerms = s.nLimitedSteps = 0;
            return r;
        })
        .def("contact_forces", [](S& s) { return v3_out(s.contactForce); })
        .def("wrenches", [](S& s) { return v3_out(s.wrench); });
    return cls;
}

// The adjoint (double and float only).
template <class T>
static void bind_adjoint(py::class_<rso::Sim<T>>& cls) {
    using S = rso::Sim<T>;
    cls
        // Reverse one frame from the current (frame-start) state; leaves the Sim at the frame end.
        .def("frame_backward", [](S& s, py::object prog, float dt, int S_, f64a gx, f64a gv, f64a glv, f64a gq) {
            std::vector<T> p;
            if (!prog.is_none()) { f64a pa = f64a::ensure(prog); p.assign(pa.data(), pa.data() + pa.size()); }
            rso::FrameGrad<T> g;
            g.init(s.n, s.R);
            v3_in(g.x, gx); v3_in(g.v, gv); v3_in(g.lv, glv); q4_in(g.q, gq);
            {
                py::gil_scoped_release rel;
                rso::FrameAdjoint<T>(s).frame_backward(p.empty() ? nullptr : p.data(), false, nullptr, nullptr, dt, S_, g);
            }
            py::dict d;
            d["x"] = v3_out(g.x); d["v"] = v3_out(g.v); d["lv"] = v3_out(g.lv); d["q"] = q4_out(g.q);
            d["P0"] = v3_out(g.P0); d["V0"] = v3_out(g.V0); d["P1"] = v3_out(g.P1);
            d["ks"] = s_out(g.ks); d["rho"] = s_out(g.rho); d["w"] = s_out(g.w);
            return d;
        });
}

// Algorithmic operation count of program-driven frames (rso::Sim<OpCount>): positions
// [N, V, 3] float32, program rows p0/v0/p1 [F, N, 3]; returns the tallies of the stepping only.
static py::dict count_program_ops(f32a positions, float density, float ks, float kb, float h, int num_itr, f32a p0,
                                  f32a v0, f32a p1, float dt, int substeps, py::object planes, float radius) {
    const int N = (int)positions.shape(0), V = (int)positions.shape(1), F = (int)p0.shape(0);
    std::vector<int> starts(N + 1);
    for (int r = 0; r <= N; r++) starts[r] = r * V;
    std::vector<uint8_t> pins((size_t)N * V, 0);
    for (int r = 0; r < N; r++) pins[(size_t)r * V] = 1;
    rso::Sim<rso::OpCount> s(positions.data(), starts.data(), N, pins.data(), density, ks, kb, h, num_itr, false, false, true,
                             0.f, 0.f);
    s.gravity = rso::V3<rso::OpCount>(0.0, 0.0, -9.81);
    s.damping = 0.0;
    s.drag = 0.0;
    if (!planes.is_none()) {
        f32a pl = f32a::ensure(planes);
        s.set_planes((int)pl.shape(0), pl.data());
        s.set_contact(radius, 0.5, 0.5, 1e-3, 2.0);
    }
    rso::op_tally().reset();
    for (int f = 0; f < F; f++)
        s.step_program(p0.data() + (size_t)f * N * 3, v0.data() + (size_t)f * N * 3, p1.data() + (size_t)f * N * 3, nullptr,
                       nullptr, dt, substeps);
    const rso::OpTally t = rso::op_tally();
    py::dict d;
    d["add"] = t.add; d["mul"] = t.mul; d["div"] = t.div; d["sqrt"] = t.sqrt; d["trans"] = t.trans; d["cmp"] = t.cmp;
    d["vertex_substeps"] = (long long)N * V * substeps * F;
    return d;
}

PYBIND11_MODULE(_oracle, m) {
    m.doc() = "CPU restatement (test oracle) of the Stable Cosserat Rods substep";
    auto c64 = bind_sim<double>(m, "Sim64");
    auto c32 = bind_sim<float>(m, "Sim32");
    bind_adjoint(c64);
    bind_adjoint(c32);
    // The op-counting instantiation: the same restated substep in double precision, every
    // floating-point operation tallied (rs_opcount.hpp) for the algorithmic FLOP figures.
    bind_sim<rso::OpCount>(m, "SimOps");
    m.def("op_tally", []() {
        const rso::OpTally t = rso::op_tally();
        py::dict d;
        d["add"] = t.add; d["mul"] = t.mul; d["div"] = t.div; d["sqrt"] = t.sqrt; d["trans"] = t.trans; d["cmp"] = t.cmp;
        return d;
    }, "operation tallies of this thread since the last op_tally_reset()");
    m.def("op_tally_reset", []() { rso::op_tally().reset(); });
    m.def("hardware_threads", []() { return (int)std::thread::hardware_concurrency(); });
    m.def("count_program_ops", &count_program_ops, py::arg("positions"), py::arg("density"), py::arg("k_stretch"),
          py::arg("k_bend"), py::arg("h"), py::arg("num_itr"), py::arg("p0"), py::arg("v0"), py::arg("p1"), py::arg("dt"),
          py::arg("substeps"), py::arg("planes") = py::none(), py::arg("radius") = 0.f);
    // FP64 brute-force mesh bake: (phi, distance, winding number), each [nx, ny, nz] float64
    m.def("bake_sdf", [](f32a verts, i32a tris, f32a origin, double spacing, std::vector<int> dims, double thickness,
                         double round, int threads) {
        rso::BakeOut o;
        {
            py::gil_scoped_release nogil;
            o = rso::bake_sdf(verts.data(), (int)verts.shape(0), tris.data(), (int)tris.shape(0), origin.data(), spacing,
                              dims[0], dims[1], dims[2], thickness, round,
                              threads > 0 ? threads : (int)std::thread::hardware_concurrency());
        }
        auto arr = [&](const std::vector<double>& v) {
            py::array_t<double> a({(py::ssize_t)dims[0], (py::ssize_t)dims[1], (py::ssize_t)dims[2]});
            std::copy(v.begin(), v.end(), a.mutable_data());
            return a;
        };
        return py::make_tuple(arr(o.phi), arr(o.dist), arr(o.wind));
    }, py::arg("vertices"), py::arg("triangles"), py::arg("origin"), py::arg("spacing"), py::arg("dims"),
       py::arg("thickness") = 0.0, py::arg("round") = 0.0, py::arg("threads") = 0);
}
