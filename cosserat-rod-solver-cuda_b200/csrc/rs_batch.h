// rs_batch.h -- host driver of one solver instance (the engine behind RopeSim / RopeBatch).
//
// Owns the caller-order host mirror, the packed device layout, the per-frame staging and the
// mesh pose machine, and launches one persistent kernel per control frame. Reference
// counterparts: ropesim::RopeBatch (csrc/batch.{h,cu}), YarnBall::Sim setup and advance
// (YarnBall.cu, sim/step.cpp) and SdfStore (csrc/sdf.{h,cu}).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "rs_types.h"

namespace rs {

// Errors surfaced through the C-ABI: invalid_argument -> RS_EINVAL, cuda_error -> RS_ECUDA,
// solver_error -> RS_ESOLVER.
struct cuda_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct solver_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct V4 {
    float x, y, z, w;
};

class Batch {
public:
    // positions: host [n, 3] in caller order (rope r owns rope_verts[r] consecutive rows);
    // pinned: host [n] (nullptr = every rope's first vertex). per_rope_env = false puts every
    // vertex in env 0 (RopeSim).
    Batch(int num_ropes, const int* rope_verts, const float* positions, const uint8_t* pinned, float density,
          float k_stretch, float k_bend, float max_h, int num_itr, bool fix_root_orientation, bool straight_rest,
          float dead_radius, float dead_barrier);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    std::mutex& mutex() { return mtx_; }

    // ---- geometry
    int num_ropes() const { return R_; }
    int num_verts() const { return n_; }
    int rope_verts(int r) const { return ustart_[r + 1] - ustart_[r]; }
    int rope_start(int r) const { return ustart_[r]; }
    bool uniform() const { return uniform_; }
    bool roots_pinned() const;

    // ---- knobs (plain writes, used by the next frame)
    float gravity[3] = {0.f, -9.8f, 0.f};
    float drag = 0.2f, drag_quad = 0.f, drag_quad_t = 0.f, damping = 1e-6f, accel = 1.f;
    int num_itr = 8;
    float max_h = 1e-3f;
    int block_override = 0;  // 0 = automatic bin size (autotuned over the first frames)
    bool sync_every_frame = true;

    // ---- host-side edits (download-modify-upload of the caller-order mirror)
    void set_vertex_inv_mass(int u, float im);
    void set_vertex_ea(int u, float ea);   // kStretch = EA * lRest (YarnBall.cu:243-244)
    void set_vertex_ei(int u, float ei);   // |qRest| = 4 EI / lRest (YarnBall.cu:250-258)
    void set_root_host(int rope, const float* pos, const float* vel, const float* q);
    void set_velocities_host(const float* vel);  // [n, 3] caller order
    void unpin_root(int rope);
    void reset_all();                       // RopeSim.reset (bindings.cpp:303-316)
    void reset_ropes(const int* ids, int count);
    void gather();
    void download(float* pos, float* vel, float* quat);  // host copies, caller order
    const std::vector<float>& inv_masses() const { return im_; }
    const std::vector<float>& rest_lengths() const { return lr_; }
    float min_seg_len() const { return min_seg_; }

    // ---- stepping
    // Root program (p0, v0, p1 [R,3]; q0, q1 [R,4] or null), caller rope order.
    void step_program(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1, float dt,
                      int substeps, bool host_inputs);
    // Constant-velocity roots (p, v [R,3]; q [R,4] or null).
    void step_legacy(const float* p, const float* v, const float* q, float dt, int substeps, bool host_inputs);
    void step_free(float dt, int substeps);
    // step_program with device inputs that calls no device allocator (see rs_batch.cpp).
    void step_program_static_scratch(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1,
                                     float dt, int substeps);
    void advance(float dt, int substeps);   // RopeSim.advance: substeps 0 = float ceil(dt / max_h)
    float time() const { return time_; }
    int last_error() const { return last_error_; }
    int bounds_violation();  // the checked build's first failed index check (status word 3)
    int last_warning() const { return last_warning_; }
    int nonfinite() const { return nonfinite_; }

    // ---- differentiable frames (no counterpart in the reference, which has no gradients).
    // Arrays are caller order (device pointers when on_device, else host): pos / vel / lvel
    // [n,3] (lvel = the velocity at the last substep's start, which the next substep's initial
    // guess extrapolates from), q [n,4]; ea / ei [n] per segment i -> i+1 (a rope's last vertex
    // is ignored), mass [n] (pinned vertices are ignored). A null pointer leaves that part alone.
    // Unlike the reference's per-vertex setters, set_parameters works between any two frames.
    void set_state(const float* pos, const float* vel, const float* lvel, const float* q, bool on_device);
    void get_state(float* pos, float* vel, float* lvel, float* q, bool on_device);
    void set_parameters(const float* ea, const float* ei, const float* mass, bool on_device);
    void get_parameters(float* ea, float* ei, float* mass, bool on_device);
    float current_h() const { return h_; }   // the last frame's substep: the next frame's lastH
    // One frame reversed: replays it from the frame-start state (io.pos ...) with the program
    // rows io.p0 / v0 / p1 (null p0 = a free frame), recording a tape, then runs the adjoint
    // kernel. All pointers are device, caller order. The batch's own state is not touched.
    // With io.tape (the tape a step_program_taped of this frame recorded) the replay is skipped;
    // io.ea / ei / mass (optional) are the frame's parameters, applied first. With synchronize
    // false the call returns with the work queued on the handle's stream.
    struct BackwardIO {
        const float *pos, *vel, *lvel, *q;
        const float *p0, *v0, *p1, *q0, *q1;
        const float *g_pos, *g_vel, *g_lvel, *g_q;
        float *o_pos, *o_vel, *o_lvel, *o_q;
        float *o_ea, *o_ei, *o_mass, *o_p0, *o_v0, *o_p1;
        const float* tape;
        const float *ea, *ei, *mass;
        const float* itape;  // iterates recorded by frame_forward (or null: recompute)
    };
    void backward(const BackwardIO& io, float dt, int substeps, float last_h, bool synchronize = true);
    // One differentiable program frame in one call: load the state and (optional) parameters,
    // step, write the end state (and the tape when given). Returns the frame's lastH.
    struct FrameIO {
        const float *pos, *vel, *lvel, *q;
        const float *ea, *ei, *mass;
        const float *p0, *v0, *p1;
        float *o_pos, *o_vel, *o_lvel, *o_q;
        float* tape;
        float* itape;  // every iterate of every substep (persistent engine, no rope-rope contact)
    };
    float frame_forward(const FrameIO& io, float dt, int substeps, bool synchronize);
    // step_program that also records the frame's substep tape (device, 16 * substeps * n
    // floats, caller order) for a later backward of this frame.
    void step_program_taped(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1,
                            float dt, int substeps, float* tape);

    // ---- views (device, caller order, stable for the object's life)
    float* out_pos() const { return d_out_pos_; }
    float* out_vel() const { return d_out_vel_; }
    float* out_q() const { return d_out_q_; }
    cudaStream_t stream() const { return stream_; }

    // ---- surface contact
    void set_contact(float radius, float mu_s, float mu_k, float v_slip, float kappa);
    void set_planes(int count, const float* rows);   // rows already unit-normalised [count, 4]
    float contact_radius() const { return c_radius_; }
    float contact_mu_s() const { return c_mu_s_; }
    float contact_mu_k() const { return c_mu_k_; }
    int add_mesh(const float* values, int nx, int ny, int nz, const float* origin, float spacing, float mu_s, float mu_k,
                 const float* pos, const float* quat, int rows);
    void set_mesh_friction(int index, float mu_s, float mu_k);
    // Targets of mesh `index` (rows 1 or R) or of every mesh (index -1, [R, M] rows).
    void set_mesh_targets(int index, const float* pos, const float* quat, int rows, const uint8_t* tele, bool tele_all,
                          bool on_device, bool tele_on_host = false);
    void clear_meshes();
    void enable_forces(bool on);
    bool forces_enabled() const { return forces_on_; }
    int num_meshes() const { return (int)grids_.size(); }
    float* contact_force_view() const { return d_force_; }
    float* wrench_view() const { return d_wrench_; }
    void contact_forces_host(float* out);   // [n, 3]
    void wrenches_host(float* out);         // [R, M, 6]

    // ---- rope-rope contact (RopeBatch::set_rope_contact, batch.cu:367-385): group_ropes
    // consecutive ropes form one contact group; groups never interact
    void set_rope_contact(bool on, float radius, float barrier, float k_collision, float mu, float k_friction,
                          float detection_scaler, int group_ropes);
    bool rope_contact() const { return rope_contact_; }

    // ---- layout introspection (tests, autotuner)
    int block() const { return block_; }
    void set_block(int block);   // 0 = automatic; repacks the device layout
    int num_bins() const { return (int)bins_.size(); }
    double last_frame_ms() const { return last_frame_ms_; }
    void set_timing(bool on) { timing_ = on; }
    // Autotuner: while on (default with an automatic bin size), the first frames run one
    // candidate bin size each (results are bitwise identical across bin sizes), then the
    // fastest is kept and remembered for this workload signature in this process.
    void set_autotune(bool on) { autotune_ = on; }
    void set_culling(bool on) { culling_ = on; }  // the persistent kernel's exact early outs
    void set_work_queue(bool on) { queue_ = on; costs_inflight_ = false; }  // the frame kernel's bin scheduling
    // Engine: 0 = one persistent launch per frame (default), 1 = the per-substep-launch plain
    // path (root, init, num_itr x (position, frame), end kernels per substep, graph-replayed).
    void set_engine(int e);
    int engine() const { return engine_; }
    bool tuning() const { return autotune_ && block_override == 0 && !tuned_; }
    const std::vector<std::pair<int, double>>& tune_log() const { return tune_log_; }

private:
    void configure(float density);
    void pack();
    void ensure_device();
    void ensure_host();
    void alloc_device();
    void stage_rows(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1, bool host);
    void run_frame(int root_mode, bool has_q0, bool has_q1, float dt, int steps, float h);
    FrameArgs frame_args(int root_mode, bool has_q0, bool has_q1, float dt, int steps) const;
    void sdf_begin();
    void sdf_end(int substeps);
    void check(cudaError_t e, const char* what);
    int pose_cache_entries() const;
    void refresh_contact_boxes();   // GridDesc::tlo/thi/never for the current contact radius
    std::vector<std::vector<float>> bmin_host_;   // per lattice: the block bounds (host copy)

    std::mutex mtx_;
    int R_ = 0, n_ = 0;
    bool uniform_ = true;
    std::vector<int> ustart_;  // [R + 1]

    // caller-order mirror: constants
    std::vector<float> im_, lr_, ks_;
    std::vector<uint32_t> fl_;
    std::vector<V4> qrest_;
    std::vector<V4> qdir_;     // unit rest rotors of construction (the direction EI scales)
    std::vector<V4> init_pos_, init_q_;
    float min_seg_ = 0.f, max_seg_ = 0.f;
    // caller-order mirror: dynamic state (valid while host_dyn_valid_)
    std::vector<V4> pos_, vel_, lvel_, q_;
    bool host_dyn_valid_ = true;   // mirror holds the latest dynamic state
    bool device_valid_ = false;    // device holds the latest state and constants
    bool layout_valid_ = false;
    bool host_const_stale_ = false; // set_parameters changed constants on the device only

    // packed layout
    int block_ = 256;
    int max_ropes_per_bin_ = 1 << 30;
    std::vector<Bin> bins_;
    std::vector<Rope> dropes_;
    std::vector<int> u2d_;   // caller vertex -> device vertex
    int max_rcount_ = 1;

    // device
    cudaStream_t stream_ = nullptr;
    Bin* d_bins_ = nullptr;
    Rope* d_ropes_ = nullptr;
    int4* d_topo_ = nullptr;
    float4 *d_pos_ = nullptr, *d_vel_ = nullptr, *d_lvel_ = nullptr, *d_q_ = nullptr, *d_qrest_ = nullptr;
    float4* d_qdir_ = nullptr;      // unit rest rotors: set_parameters scales these (idempotent)
    float4 *d_init_pos_ = nullptr, *d_init_q_ = nullptr;
    float *d_out_pos_ = nullptr, *d_out_vel_ = nullptr, *d_out_q_ = nullptr;
    float* d_prog_ = nullptr;       // [R, 17]
    float* h_prog_ = nullptr;       // pinned staging [R, 17]
    int* d_status_ = nullptr;       // [4]
    int* h_status_ = nullptr;       // pinned [4]
    int2* d_ranges_ = nullptr;      // [R] reset ranges
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    // the frame kernel's work queue (frame_kernel): counter, bin order (longest measured first),
    // per-bin times of the last frame (device and pinned host copies)
    bool queue_ = true;
    int* d_queue_ = nullptr;
    int* d_order_ = nullptr;
    float* d_bin_cost_ = nullptr;
    float* h_bin_cost_ = nullptr;
    int* h_order_ = nullptr;
    std::vector<int> order_scratch_;
    bool costs_inflight_ = false;
    cudaEvent_t ev_cost_ = nullptr;
    void reorder_bins();
    bool timing_ = false;
    double last_frame_ms_ = 0.0;
    bool autotune_ = true, tuned_ = false;
    bool culling_ = true;
    int engine_ = 0;
    // rope-rope contact
    bool rope_contact_ = false;
    float rc_radius_ = 1e-4f, rc_barrier_ = 8e-4f, rc_kcol_ = 1e-5f, rc_mu_ = 0.1f, rc_kfric_ = 5.f, rc_scaler_ = 1.2f;
    int group_ropes_ = 1;
    int max_unit_verts_ = 0;
    bool oversize_ = false;          // a contact group is larger than one CTA: plain engine
    std::vector<int4> grp_;          // host copy of d_grp_
    int4* d_grp_ = nullptr;          // [n] (group start, group end, rope start, rope end), device order
    int* d_cols_ = nullptr;          // [kMaxCols * n] candidate lists (scratch)
    int* d_ncols_ = nullptr;         // [n]
    float* d_maxstep_ = nullptr;     // [n]
    float* d_pad_ = nullptr;         // [n]
    PlainBufs pl_{};
    FrameArgs* d_pl_args_ = nullptr;
    FrameArgs* h_pl_args_ = nullptr;   // pinned staging of the frame parameters
    cudaGraphExec_t pl_graph_ = nullptr;
    std::string pl_graph_key_;
    void plain_alloc();
    void run_frame_plain(const FrameArgs& a);
    std::vector<int> tune_cands_;
    std::vector<std::pair<int, double>> tune_log_;
    int tune_block_ = 0;            // bin size chosen by the autotuner (0 = none yet)
    void tune_before_frame();
    void tune_after_frame();
    std::string tune_key() const;

    // solver bookkeeping (YarnBall MetaData)
    float h_ = 1e-3f, last_h_ = 1e-3f, time_ = 0.f;
    int last_error_ = 0, last_warning_ = 0, nonfinite_ = 0;

    // contact material and planes
    int num_planes_ = 0;
    float planes_[kMaxPlanes][4] = {};
    float c_radius_ = 0.f, c_kappa_ = 2.f, c_mu_s_ = 0.f, c_mu_k_ = 0.f, c_vslip_ = 1e-3f;

    // meshes (sdf.h)
    std::vector<GridDesc> grids_;
    std::vector<float> boxes_;      // [M, 6] object-frame lattice boxes
    float* d_boxes_ = nullptr;      // [64, 6]
    Pose7 *d_cur_ = nullptr, *d_tgt_ = nullptr;
    uint8_t* d_tele_ = nullptr;
    Motion* d_motion_ = nullptr;
    Pose* d_poses_ = nullptr;
    float* d_stage_ = nullptr;      // [R * 64 * 7] host-call staging
    uint8_t* d_stage_tele_ = nullptr;
    bool pending_set_ = false, moving_ = false, sdf_moving_ = false, forces_on_ = false;
    float* d_force_ = nullptr;      // [n, 3]
    float* d_wrench_ = nullptr;     // [R, 64, 6]
    int last_substeps_ = 1;

    // differentiable frames: replay state, staging and the substep tape
    float4 *gs_pos_ = nullptr, *gs_vel_ = nullptr, *gs_lvel_ = nullptr, *gs_q_ = nullptr;
    float* gs_buf_ = nullptr;       // [13 n] host-call staging / replay views
    float4* d_tape_ = nullptr;      // [tape_steps_][4][n]
    int tape_steps_ = 0;
    float4* pending_tape_ = nullptr;  // tape of the frame being launched (step_program_taped)
    float4* pending_itape_ = nullptr; // iterate tape of the frame being launched (frame_forward)
    bool itape_usable() const { return engine_ == 0 && !rope_contact_; }
    void grad_alloc(int substeps);
    // the per-launch adjoint (contact groups larger than one CTA, plain engine)
    float4* d_padj_ = nullptr;      // adjoint_plain_words(n, iters) float4
    size_t padj_words_ = 0;
    FrameArgs* d_adj_args_ = nullptr;
    FrameArgs* h_adj_args_ = nullptr;  // pinned staging of the backward's frame parameters
    // grid broad phase of contact groups larger than one CTA (null until first needed)
    RopeGrid grid_{};
    void* grid_mem_ = nullptr;
    const RopeGrid* rope_grid();
};

}  // namespace rs
