// rs_capi.cpp -- the extern "C" boundary (include/ropesim_b200.h) over rs::Batch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/ropesim_b200.h"
#include "rs_batch.h"
#include "rs_kernels.h"

struct rs_batch {
    rs::Batch* impl;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        f();
        return RS_OK;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return RS_EINVAL;
    } catch (const rs::cuda_error& e) {
        g_last_error = e.what();
        return RS_ECUDA;
    } catch (const rs::solver_error& e) {
        g_last_error = e.what();
        return RS_ESOLVER;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return RS_ECUDA;
    } catch (...) {
        g_last_error = "unknown error";
        return RS_ECUDA;
    }
}

void need(bool ok, const char* msg) {
    if (!ok) throw std::invalid_argument(msg);
}

rs::Batch& B(rs_batch* b) {
    need(b && b->impl, "null rs_batch handle");
    return *b->impl;
}

}  // namespace

extern "C" {

const char* rs_last_error_string(void) { return g_last_error.c_str(); }
const char* rs_version(void) { return "ropesim_b200 0.1 (sm_100a)"; }

int rs_batch_create(rs_batch** out, int num_ropes, const int* rope_verts, const float* positions, const uint8_t* pinned,
                    float density, float k_stretch, float k_bend, float max_h, int num_itr, int fix_root_orientation,
                    int straight_rest, float dead_radius, float dead_barrier) {
    return guarded([&] {
        need(out && rope_verts && positions, "null argument");
        need(num_ropes >= 1, "num_ropes must be >= 1");
        need(density > 0 && k_stretch > 0 && k_bend > 0 && max_h > 0 && num_itr >= 1,
             "density, k_stretch, k_bend, max_h > 0 and num_itr >= 1 required");
        rs::Batch* impl = new rs::Batch(num_ropes, rope_verts, positions, pinned, density, k_stretch, k_bend, max_h, num_itr,
                                        fix_root_orientation != 0, straight_rest != 0, dead_radius, dead_barrier);
        *out = new rs_batch{impl};
    });
}

int rs_batch_create_straight(rs_batch** out, int num_ropes, int verts_per_rope, const float* root_pos, float seg_len,
                             const float* dir3, float density, float k_stretch, float k_bend, float max_h, int num_itr,
                             int fix_root_orientation, float dead_radius, float dead_barrier) {
    return guarded([&] {
        need(out && root_pos && dir3, "null argument");
        need(num_ropes >= 1 && verts_per_rope >= 3, "num_envs >= 1 and verts_per_rope >= 3 required");
        need(seg_len > 0, "seg_len must be > 0");
        const float l2 = (dir3[0] * dir3[0] + dir3[1] * dir3[1]) + dir3[2] * dir3[2];
        need(std::sqrt(l2) > 0, "dir must be nonzero");
        // glm::normalize(dir) = dir * (1 / sqrt(dot)), batch.cu:343
        const float inv = 1.f / std::sqrt(l2);
        const float d[3] = {dir3[0] * inv, dir3[1] * inv, dir3[2] * inv};
        std::vector<float> pos((size_t)num_ropes * verts_per_rope * 3);
        for (int e = 0; e < num_ropes; e++)
            for (int v = 0; v < verts_per_rope; v++)
                for (int k = 0; k < 3; k++)
                    pos[((size_t)e * verts_per_rope + v) * 3 + k] = root_pos[3 * e + k] + (float(v) * seg_len) * d[k];
        std::vector<int> verts(num_ropes, verts_per_rope);
        need(density > 0 && k_stretch > 0 && k_bend > 0 && max_h > 0 && num_itr >= 1,
             "density, k_stretch, k_bend, max_h > 0 and num_itr >= 1 required");
        rs::Batch* impl = new rs::Batch(num_ropes, verts.data(), pos.data(), nullptr, density, k_stretch, k_bend, max_h,
                                        num_itr, fix_root_orientation != 0, false, dead_radius, dead_barrier);
        *out = new rs_batch{impl};
    });
}

int rs_batch_destroy(rs_batch* b) {
    return guarded([&] {
        if (!b) return;
        delete b->impl;
        delete b;
    });
}

int rs_batch_set_param(rs_batch* b, int which, float value) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        switch (which) {
            case RS_P_DRAG: s.drag = value; break;
            case RS_P_DRAG_QUAD:
                need(std::isfinite(value) && value >= 0, "drag_quad must be finite and >= 0");
                s.drag_quad = value;
                break;
            case RS_P_DRAG_QUAD_T:
                need(std::isfinite(value) && value >= 0, "drag_quad_t must be finite and >= 0");
                s.drag_quad_t = value;
                break;
            case RS_P_DAMPING: s.damping = value; break;
            case RS_P_ACCEL: s.accel = value; break;
            case RS_P_MAX_H:
                need(value > 0, "max_h must be > 0");
                s.max_h = value;
                break;
            default: throw std::invalid_argument("unknown or read-only parameter");
        }
    });
}

int rs_batch_get_param(rs_batch* b, int which, float* value) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(value != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        switch (which) {
            case RS_P_DRAG: *value = s.drag; break;
            case RS_P_DRAG_QUAD: *value = s.drag_quad; break;
            case RS_P_DRAG_QUAD_T: *value = s.drag_quad_t; break;
            case RS_P_DAMPING: *value = s.damping; break;
            case RS_P_ACCEL: *value = s.accel; break;
            case RS_P_MAX_H: *value = s.max_h; break;
            case RS_P_TIME: *value = s.time(); break;
            case RS_P_H: *value = s.current_h(); break;
            default: throw std::invalid_argument("unknown parameter");
        }
    });
}

int rs_batch_set_num_itr(rs_batch* b, int num_itr) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(num_itr >= 1, "num_itr must be >= 1");
        std::lock_guard<std::mutex> g(s.mutex());
        s.num_itr = num_itr;
    });
}
int rs_batch_get_num_itr(rs_batch* b, int* num_itr) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(num_itr != nullptr, "null argument");
        *num_itr = s.num_itr;
    });
}
int rs_batch_set_gravity(rs_batch* b, const float* g3) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(g3 != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        for (int k = 0; k < 3; k++) s.gravity[k] = g3[k];
    });
}
int rs_batch_get_gravity(rs_batch* b, float* g3) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(g3 != nullptr, "null argument");
        for (int k = 0; k < 3; k++) g3[k] = s.gravity[k];
    });
}
int rs_batch_set_block(rs_batch* b, int block) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(block == 0 || block == 64 || block == 128 || block == 256 || block == 512 || block == 1024,
             "block must be 0, 64, 128, 256, 512 or 1024");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_block(block);
    });
}
int rs_batch_layout(rs_batch* b, int* block, int* num_bins) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (block) *block = s.block();
        if (num_bins) *num_bins = s.num_bins();
    });
}
int rs_batch_set_autotune(rs_batch* b, int on) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_autotune(on != 0);
    });
}
int rs_batch_set_culling(rs_batch* b, int on) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_culling(on != 0);
    });
}
int rs_batch_set_work_queue(rs_batch* b, int on) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_work_queue(on != 0);
    });
}
int rs_batch_set_engine(rs_batch* b, int engine) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_engine(engine);
    });
}
int rs_batch_set_sync(rs_batch* b, int every_frame) {
    return guarded([&] {
        rs::Batch& s = B(b);
        s.sync_every_frame = every_frame != 0;
    });
}

int rs_batch_num_verts(rs_batch* b, int* n, int* num_ropes) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (n) *n = s.num_verts();
        if (num_ropes) *num_ropes = s.num_ropes();
    });
}
int rs_batch_rope_verts(rs_batch* b, int* rope_verts) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(rope_verts != nullptr, "null argument");
        for (int r = 0; r < s.num_ropes(); r++) rope_verts[r] = s.rope_verts(r);
    });
}
int rs_batch_download(rs_batch* b, float* pos, float* vel, float* quat) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.download(pos, vel, quat);
    });
}
int rs_batch_inv_masses(rs_batch* b, float* out) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(out != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        std::memcpy(out, s.inv_masses().data(), sizeof(float) * s.num_verts());
    });
}
int rs_batch_rest_lengths(rs_batch* b, float* out) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(out != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        std::memcpy(out, s.rest_lengths().data(), sizeof(float) * s.num_verts());
    });
}
int rs_batch_min_segment(rs_batch* b, float* out) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(out != nullptr, "null argument");
        *out = s.min_seg_len();
    });
}
int rs_batch_set_masses(rs_batch* b, const float* m) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(m != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        const auto& im = s.inv_masses();
        for (int u = 0; u < s.num_verts(); u++)
            need(im[u] == 0.f || (std::isfinite(m[u]) && m[u] > 0), "node masses must be finite and > 0 (pinned columns ignored)");
        for (int u = 0; u < s.num_verts(); u++)
            if (im[u] != 0.f) s.set_vertex_inv_mass(u, 1.f / m[u]);
    });
}
static void check_last_vertex_ignored(rs::Batch& s, const float* a, const char* msg) {
    for (int r = 0; r < s.num_ropes(); r++)
        for (int i = 0; i + 1 < s.rope_verts(r); i++) {
            const float v = a[s.rope_start(r) + i];
            need(std::isfinite(v) && v > 0, msg);
        }
}
int rs_batch_set_stretch_stiffnesses(rs_batch* b, const float* ea) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(ea != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        check_last_vertex_ignored(s, ea, "EA values must be finite and > 0");
        for (int r = 0; r < s.num_ropes(); r++)
            for (int i = 0; i + 1 < s.rope_verts(r); i++) s.set_vertex_ea(s.rope_start(r) + i, ea[s.rope_start(r) + i]);
    });
}
int rs_batch_set_bend_stiffnesses(rs_batch* b, const float* ei) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(ei != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        check_last_vertex_ignored(s, ei, "EI values must be finite and > 0");
        for (int r = 0; r < s.num_ropes(); r++)
            for (int i = 0; i + 1 < s.rope_verts(r); i++) s.set_vertex_ei(s.rope_start(r) + i, ei[s.rope_start(r) + i]);
    });
}
int rs_batch_set_velocities(rs_batch* b, const float* vel) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(vel != nullptr, "null argument");
        for (int i = 0; i < 3 * s.num_verts(); i++) need(std::isfinite(vel[i]), "velocities must be finite");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_velocities_host(vel);
    });
}
int rs_batch_set_root(rs_batch* b, int rope, const float* pos3, const float* vel3, const float* q4) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(pos3 && vel3, "null argument");
        need(rope >= 0 && rope < s.num_ropes(), "rope index out of range");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_root_host(rope, pos3, vel3, q4);
    });
}
int rs_batch_unpin_root(rs_batch* b, int rope) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(rope >= 0 && rope < s.num_ropes(), "rope index out of range");
        std::lock_guard<std::mutex> g(s.mutex());
        s.unpin_root(rope);
    });
}
int rs_batch_roots_pinned(rs_batch* b, int* pinned) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(pinned != nullptr, "null argument");
        *pinned = s.roots_pinned() ? 1 : 0;
    });
}

int rs_batch_step_program(rs_batch* b, const float* p0, const float* v0, const float* p1, const float* q0, const float* q1,
                          float dt, int substeps, int on_host) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(p0 && v0 && p1, "null argument");
        need(dt > 0, "dt must be > 0");
        need(substeps >= 1, "substeps must be >= 1");
        need(!(q1 && !q0), "root_q_end requires root_q");
        std::lock_guard<std::mutex> g(s.mutex());
        s.step_program(p0, v0, p1, q0, q1, dt, substeps, on_host != 0);
    });
}
int rs_batch_step_program_static_scratch(rs_batch* b, const float* p0, const float* v0, const float* p1, const float* q0,
                                         const float* q1, float dt, int substeps) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(p0 && v0 && p1, "null argument");
        need(dt > 0, "dt must be > 0");
        need(substeps >= 1, "substeps must be >= 1");
        need(!(q1 && !q0), "root_q_end requires root_q");
        std::lock_guard<std::mutex> g(s.mutex());
        s.step_program_static_scratch(p0, v0, p1, q0, q1, dt, substeps);
    });
}

int rs_batch_step_legacy(rs_batch* b, const float* p, const float* v, const float* q, float dt, int substeps, int on_host) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(p && v, "null argument");
        need(dt > 0, "dt must be > 0");
        need(substeps >= 1, "substeps must be >= 1");
        std::lock_guard<std::mutex> g(s.mutex());
        s.step_legacy(p, v, q, dt, substeps, on_host != 0);
    });
}
int rs_batch_step_free(rs_batch* b, float dt, int substeps) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(dt > 0 && substeps >= 1, "dt > 0 and substeps >= 1 required");
        std::lock_guard<std::mutex> g(s.mutex());
        s.step_free(dt, substeps);
    });
}
int rs_batch_advance(rs_batch* b, float dt, int substeps) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(substeps >= 0, "substeps must be >= 0");
        std::lock_guard<std::mutex> g(s.mutex());
        s.advance(dt, substeps);
    });
}
int rs_batch_reset_ropes(rs_batch* b, const int* ids, int count) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(count >= 0 && (count == 0 || ids), "bad ids");
        need(count <= s.num_ropes(), "ids longer than num_envs");
        for (int i = 0; i < count; i++) need(ids[i] >= 0 && ids[i] < s.num_ropes(), "env id out of range");
        std::lock_guard<std::mutex> g(s.mutex());
        s.reset_ropes(ids, count);
    });
}
int rs_batch_reset_all(rs_batch* b) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.reset_all();
    });
}
int rs_batch_gather(rs_batch* b) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.gather();
    });
}
int rs_batch_views(rs_batch* b, float** pos, float** vel, float** quat) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (pos) *pos = s.out_pos();
        if (vel) *vel = s.out_vel();
        if (quat) *quat = s.out_q();
    });
}
int rs_batch_status(rs_batch* b, int* last_error, int* last_warning, int* nonfinite) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (last_error) *last_error = s.last_error();
        if (last_warning) *last_warning = s.last_warning();
        if (nonfinite) *nonfinite = s.nonfinite();
    });
}
int rs_batch_bounds_check(rs_batch* b, int* code, int* checked) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        if (code) *code = s.bounds_violation();
        if (checked) *checked = rs::kChecked ? 1 : 0;
    });
}
int rs_batch_stream(rs_batch* b, void** stream) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(stream != nullptr, "null argument");
        *stream = (void*)s.stream();
    });
}
int rs_batch_set_timing(rs_batch* b, int on) {
    return guarded([&] {
        rs::Batch& s = B(b);
        s.set_timing(on != 0);
    });
}
int rs_batch_last_frame_ms(rs_batch* b, double* ms) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(ms != nullptr, "null argument");
        *ms = s.last_frame_ms();
    });
}

int rs_batch_set_contact(rs_batch* b, float radius, float mu_s, float mu_k, float v_slip, float kappa) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(radius > 0 && kappa > 0 && mu_s >= 0 && mu_k >= 0 && v_slip > 0,
             "surface contact needs radius > 0, kappa > 0, mu_s >= 0, mu_k >= 0, v_slip > 0");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_contact(radius, mu_s, mu_k, v_slip, kappa);
    });
}
int rs_batch_get_contact(rs_batch* b, float* radius, float* mu_s, float* mu_k) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (radius) *radius = s.contact_radius();
        if (mu_s) *mu_s = s.contact_mu_s();
        if (mu_k) *mu_k = s.contact_mu_k();
    });
}
int rs_batch_set_planes(rs_batch* b, int count, const float* rows) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(count >= 0 && count <= rs::kMaxPlanes, "planes must be [P<=8, 4] rows (nx, ny, nz, w): half-spaces n.x >= w");
        need(count == 0 || rows, "null argument");
        std::vector<float> unit(4 * (size_t)count);
        for (int i = 0; i < count; i++) {
            const float nx = rows[4 * i], ny = rows[4 * i + 1], nz = rows[4 * i + 2], w = rows[4 * i + 3];
            const float l = std::sqrt((nx * nx + ny * ny) + nz * nz);
            need(l > 0 && std::isfinite(l) && std::isfinite(w), "plane rows need a finite, nonzero normal and a finite offset");
            unit[4 * i] = nx / l; unit[4 * i + 1] = ny / l; unit[4 * i + 2] = nz / l; unit[4 * i + 3] = w / l;
        }
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_planes(count, unit.data());
    });
}
int rs_batch_set_rope_contact(rs_batch* b, int enabled, float radius, float barrier, float k_collision, float mu,
                              float k_friction, float detection_scaler, int group_ropes) {
    return guarded([&] {
        rs::Batch& s = B(b);
        if (enabled)
            need(radius > 0 && barrier > 0 && k_collision > 0 && mu >= 0 && k_friction >= 0 && detection_scaler > 1 &&
                     group_ropes >= 1,
                 "rope contact needs radius, barrier, k_collision > 0, mu, k_friction >= 0, detection_scaler > 1, "
                 "group_ropes >= 1");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_rope_contact(enabled != 0, radius, barrier, k_collision, mu, k_friction, detection_scaler, group_ropes);
    });
}

int rs_batch_add_mesh(rs_batch* b, const float* values, int nx, int ny, int nz, const float* origin3, float spacing,
                      float mu_s, float mu_k, const float* pos, const float* quat, int rows, int* index) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(values && origin3 && pos && quat && index, "null argument");
        need(nx >= 2 && ny >= 2 && nz >= 2, "sdf values must be [nx, ny, nz] with every dim >= 2");
        need(spacing > 0 && std::isfinite(spacing), "sdf spacing must be > 0");
        need(rows == 1 || rows == s.num_ropes(), "pose rows must be 1 or num_envs");
        need(mu_s >= 0 && mu_k >= 0, "mu_s / mu_k must be >= 0");
        const size_t cnt = (size_t)nx * ny * nz;
        for (size_t i = 0; i < cnt; i++) need(std::isfinite(values[i]), "sdf values must be finite");
        std::lock_guard<std::mutex> g(s.mutex());
        need(s.contact_radius() > 0, "set the contact material first: set_contact(radius, ...) or set_planes(..., radius=)");
        *index = s.add_mesh(values, nx, ny, nz, origin3, spacing, mu_s, mu_k, pos, quat, rows);
    });
}
int rs_batch_set_mesh_friction(rs_batch* b, int index, float mu_s, float mu_k) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(mu_s >= 0 && mu_k >= 0, "mu_s / mu_k must be >= 0");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_mesh_friction(index, mu_s, mu_k);
    });
}
int rs_batch_set_mesh_poses(rs_batch* b, int index, const float* pos, const float* quat, int rows, const uint8_t* tele,
                            int tele_all, int on_device) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(pos && quat, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_mesh_targets(index, pos, quat, rows, tele, tele_all != 0, (on_device & 1) != 0, (on_device & 2) != 0);
    });
}
int rs_batch_clear_meshes(rs_batch* b) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.clear_meshes();
    });
}
int rs_batch_num_meshes(rs_batch* b, int* count) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(count != nullptr, "null argument");
        *count = s.num_meshes();
    });
}
int rs_batch_enable_contact_forces(rs_batch* b, int on) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.enable_forces(on != 0);
    });
}
int rs_batch_contact_forces(rs_batch* b, float* out) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(out != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        s.contact_forces_host(out);
    });
}
int rs_batch_mesh_wrenches(rs_batch* b, float* out) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(out != nullptr, "null argument");
        std::lock_guard<std::mutex> g(s.mutex());
        s.wrenches_host(out);
    });
}
int rs_batch_contact_views(rs_batch* b, float** forces, float** wrenches) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(s.forces_enabled(), "enable_contact_forces(True) first");
        if (forces) *forces = s.contact_force_view();
        if (wrenches) *wrenches = s.wrench_view();
    });
}

// ------------------------------------------------------------------ differentiable frames
int rs_batch_set_state(rs_batch* b, const float* pos, const float* vel, const float* lvel, const float* q, int on_device) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_state(pos, vel, lvel, q, on_device != 0);
    });
}
int rs_batch_get_state(rs_batch* b, float* pos, float* vel, float* lvel, float* q, int on_device) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.get_state(pos, vel, lvel, q, on_device != 0);
    });
}
int rs_batch_set_parameters(rs_batch* b, const float* ea, const float* ei, const float* mass, int on_device) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.set_parameters(ea, ei, mass, on_device != 0);
    });
}
int rs_batch_get_parameters(rs_batch* b, float* ea, float* ei, float* mass, int on_device) {
    return guarded([&] {
        rs::Batch& s = B(b);
        std::lock_guard<std::mutex> g(s.mutex());
        s.get_parameters(ea, ei, mass, on_device != 0);
    });
}
static int backward_impl(rs_batch* b, const rs_backward_io* io, float dt, int substeps, float last_h, bool sync) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(io != nullptr, "null argument");
        rs::Batch::BackwardIO x{io->pos, io->vel, io->lvel, io->q, io->p0, io->v0, io->p1, io->q0, io->q1,
                                io->g_pos, io->g_vel, io->g_lvel, io->g_q, io->o_pos, io->o_vel, io->o_lvel, io->o_q,
                                io->o_ea, io->o_ei, io->o_mass, io->o_p0, io->o_v0, io->o_p1, io->tape,
                                io->ea, io->ei, io->mass, io->itape};
        std::lock_guard<std::mutex> g(s.mutex());
        s.backward(x, dt, substeps, last_h, sync);
    });
}
int rs_batch_backward(rs_batch* b, const rs_backward_io* io, float dt, int substeps, float last_h) {
    return backward_impl(b, io, dt, substeps, last_h, true);
}
int rs_batch_backward_async(rs_batch* b, const rs_backward_io* io, float dt, int substeps, float last_h) {
    return backward_impl(b, io, dt, substeps, last_h, false);
}
int rs_batch_frame_forward(rs_batch* b, const rs_frame_io* io, float dt, int substeps, float* last_h) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(io != nullptr, "null argument");
        rs::Batch::FrameIO x{io->pos, io->vel, io->lvel, io->q, io->ea, io->ei, io->mass, io->p0, io->v0, io->p1,
                             io->out_pos, io->out_vel, io->out_lvel, io->out_q, io->tape, io->itape};
        std::lock_guard<std::mutex> g(s.mutex());
        const float lh = s.frame_forward(x, dt, substeps, false);
        if (last_h) *last_h = lh;
    });
}
int rs_batch_step_program_taped(rs_batch* b, const float* p0, const float* v0, const float* p1, const float* q0,
                                const float* q1, float dt, int substeps, float* tape) {
    return guarded([&] {
        rs::Batch& s = B(b);
        need(p0 && v0 && p1 && tape, "null argument");
        need(dt > 0, "dt must be > 0");
        need(substeps >= 1, "substeps must be >= 1");
        need(!(q1 && !q0), "root_q_end requires root_q");
        std::lock_guard<std::mutex> g(s.mutex());
        s.step_program_taped(p0, v0, p1, q0, q1, dt, substeps, tape);
    });
}

int rs_sdf_bake(const float* vertices, int num_vertices, const int* triangles, int num_triangles, const float* origin3,
                double spacing, int nx, int ny, int nz, float thickness, float round, float* out, int out_on_device,
                void* stream, unsigned long long* counters) {
    return guarded([&] {
        need(vertices && triangles && origin3 && out, "null argument");
        std::string err;
        const cudaError_t e = rs::sdf_bake(vertices, num_vertices, triangles, num_triangles, origin3, spacing, nx, ny, nz,
                                           thickness, round, out, out_on_device != 0, counters,
                                           static_cast<cudaStream_t>(stream), &err);
        if (e == cudaErrorInvalidValue && !err.empty() && err.rfind("sdf bake:", 0) != 0) throw std::invalid_argument(err);
        if (e != cudaSuccess) throw rs::cuda_error(err.empty() ? cudaGetErrorString(e) : err);
    });
}

int rs_probe_fp32_peak(double* tflops, double* ms) {
    return guarded([&] {
        need(tflops != nullptr, "null argument");
        int dev = 0, sms = 0;
        auto chk = [](cudaError_t e, const char* w) { if (e != cudaSuccess) throw rs::cuda_error(std::string(w) + ": " + cudaGetErrorString(e)); };
        chk(cudaGetDevice(&dev), "cudaGetDevice");
        chk(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
        float* out = nullptr;
        const int threads = 256, blocks = sms * 8, iters = 4096;
        chk(cudaMalloc(&out, sizeof(float) * threads * blocks), "cudaMalloc(probe)");
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        float best = 1e30f;
        for (int rep = 0; rep < 5; rep++) {
            cudaEventRecord(a, 0);
            chk(rs::launch_fp32_probe(out, blocks, threads, iters, 0), "probe");
            cudaEventRecord(b, 0);
            chk(cudaEventSynchronize(b), "probe sync");
            float t = 0.f;
            cudaEventElapsedTime(&t, a, b);
            if (rep > 0) best = std::min(best, t);
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaFree(out);
        const double flops = 2.0 * 16 * 8 * (double)iters * threads * blocks;
        *tflops = flops / (best * 1e-3) / 1e12;
        if (ms) *ms = best;
    });
}

}  // extern "C"
