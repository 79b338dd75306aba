/* ropesim_b200.h -- C-ABI of the B200 Stable Cosserat Rods substep engine.
 *
 * The boundary the reference's Python module binds (csrc/bindings.cpp of
 * DeformX/Cosserat-Rod-Solver-CUDA, pybind11 `_ropesim`) is re-expressed as plain C: opaque
 * handles, host or device float pointers with explicit sizes, `int` status codes and a
 * thread-local error string. No torch or pybind11 types cross it. The pybind11 module
 * `ropesim._ropesim` of this repository is one client; ctypes / cffi clients work the same way
 * (load libropesim_b200.so, declare these signatures, pass device addresses as integers).
 *
 * Layout conventions: "caller order" is the reference's flat order (rope r owns its vertices
 * consecutively, ropes in index order). Rotors are (x, y, z, w). All device pointers are
 * float32, C-contiguous. Every call is serialised by a per-handle mutex; device work runs on
 * the handle's own blocking stream (ordered with the legacy default stream, as the
 * reference's solver stream is: csrc/batch.h:9-14).
 */
#ifndef ROPESIM_B200_H
#define ROPESIM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define RS_API __declspec(dllexport)
#else
#define RS_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. RS_EINVAL maps to the reference's ValueError (bindings.cpp throws
 * py::value_error before any state change), RS_ECUDA to its RuntimeError (Common.h:17-30),
 * RS_ESOLVER to Sim::checkErrors' solver errors (YarnBall.cu:311-339). */
#define RS_OK 0
#define RS_EINVAL 1
#define RS_ECUDA 2
#define RS_ESOLVER 3

typedef struct rs_batch rs_batch;

/* Last error message of the calling thread ("" when none). */
RS_API const char* rs_last_error_string(void);
/* Library version string. */
RS_API const char* rs_version(void);

/* ---------------------------------------------------------------- construction
 * Replaces RopeBatch::RopeBatch + Sim::configure/setKStretch/setKBend (csrc/batch.cu:193-276,
 * YarnBall.cu:112-259) and RopeSim::RopeSim (bindings.cpp:196-265).
 * rope_verts[num_ropes] (each >= 3, <= 1024; uneven lengths allowed), positions host
 * [sum(rope_verts), 3], pinned host [sum(rope_verts)] or NULL (each rope's first vertex).
 * dead_radius / dead_barrier: the rope-rope radii used only by the segment-length validity
 * check (batch.cu:363-375: 0.01 / 0.08 of the shortest segment). */
RS_API int rs_batch_create(rs_batch** out, int num_ropes, const int* rope_verts, const float* positions,
                    const uint8_t* pinned, float density, float k_stretch, float k_bend, float max_h,
                    int num_itr, int fix_root_orientation, int straight_rest, float dead_radius,
                    float dead_barrier);
/* Straight ropes from roots (RopeBatch(num_envs, verts_per_rope, root_pos, seg_len, dir, ...),
 * bindings.cpp:736-767 / batch.cu:343-350): vertex v of rope e at root_e + v * seg_len * dir. */
RS_API int rs_batch_create_straight(rs_batch** out, int num_ropes, int verts_per_rope, const float* root_pos,
                             float seg_len, const float* dir3, float density, float k_stretch, float k_bend,
                             float max_h, int num_itr, int fix_root_orientation, float dead_radius,
                             float dead_barrier);
RS_API int rs_batch_destroy(rs_batch* b);

/* ---------------------------------------------------------------- knobs (MetaData fields)
 * Replaces the property setters/getters of bindings.cpp:535-579 and :860-886. */
enum rs_param {
    RS_P_DRAG = 0,        /* linear velocity decay [1/s]            (meta.drag) */
    RS_P_DRAG_QUAD = 1,   /* quadratic normal drag [1/m]            (meta.dragQuad) */
    RS_P_DRAG_QUAD_T = 2, /* quadratic tangential drag [1/m]        (meta.dragQuadT) */
    RS_P_DAMPING = 3,     /* YarnBall damping (enters as damping/h) (meta.damping) */
    RS_P_ACCEL = 4,       /* local-solve relaxation                 (meta.accelerationRatio) */
    RS_P_MAX_H = 5,       /* largest substep of advance()           (Sim::maxH) */
    RS_P_TIME = 6,        /* read-only accumulated time             (meta.time) */
    RS_P_H = 7            /* read-only substep of the last frame    (meta.h; the next frame's lastH) */
};
RS_API int rs_batch_set_param(rs_batch* b, int which, float value);
RS_API int rs_batch_get_param(rs_batch* b, int which, float* value);
RS_API int rs_batch_set_num_itr(rs_batch* b, int num_itr);
RS_API int rs_batch_get_num_itr(rs_batch* b, int* num_itr);
RS_API int rs_batch_set_gravity(rs_batch* b, const float* g3);
RS_API int rs_batch_get_gravity(rs_batch* b, float* g3);
/* Bin size (CTA threads) of the packed layout; 0 = automatic. Used by the autotuner. */
RS_API int rs_batch_set_block(rs_batch* b, int block);
RS_API int rs_batch_layout(rs_batch* b, int* block, int* num_bins);
/* Bin-size autotuner (default on while the bin size is automatic): the first frames each run
 * one candidate bin size, then the fastest is kept (results are bitwise identical across bin
 * sizes) and remembered per workload signature for the process. */
RS_API int rs_batch_set_autotune(rs_batch* b, int on);
/* The persistent kernel's exact early outs (default on): per substep, the iterate displacement
 * below which no plane and no candidate lattice can be reached (Lipschitz bound of the trilinear
 * field), per lattice the world box of the blocks that can reach the contact radius, and the
 * blocks whose lower bound clears it. They only skip evaluations whose gap is >= 0, so results
 * are bitwise the same either way; off evaluates every surface at every iteration, as the
 * reference does (for checking that claim). No counterpart in the reference. */
RS_API int rs_batch_set_culling(rs_batch* b, int on);
/* Bin scheduling of the frame kernel (default on): resident CTAs take bins from a work queue in
 * longest-first order of the previous frame's measured bin times (measured when the step reads
 * its status every frame); off launches one CTA per bin in packing order. Results are bitwise
 * the same either way. No counterpart in the reference (its substep launches per kernel). */
RS_API int rs_batch_set_work_queue(rs_batch* b, int on);
/* Engine: 0 = one persistent kernel per control frame (default); 1 = the per-substep-launch
 * plain path (the reference's launch structure: root, init, num_itr x (position, frame), end
 * kernels per substep, the iterations replayed from a CUDA graph), the in-repo baseline. */
RS_API int rs_batch_set_engine(rs_batch* b, int engine);
/* 1 (default) = synchronise and read the status words after every frame (checkErrors). */
RS_API int rs_batch_set_sync(rs_batch* b, int every_frame);

/* ---------------------------------------------------------------- geometry / host state
 * Replaces RopeSim's host getters and setters (bindings.cpp:303-462, :525-532) and RopeBatch's
 * per-vertex property API (bindings.cpp:1109-1201). Arrays are caller order. */
RS_API int rs_batch_num_verts(rs_batch* b, int* n, int* num_ropes);
RS_API int rs_batch_rope_verts(rs_batch* b, int* rope_verts /* [num_ropes] */);
RS_API int rs_batch_download(rs_batch* b, float* pos /*[n,3] or NULL*/, float* vel /*[n,3] or NULL*/,
                      float* quat /*[n,4] or NULL*/);
RS_API int rs_batch_inv_masses(rs_batch* b, float* out /* [n] */);
RS_API int rs_batch_rest_lengths(rs_batch* b, float* out /* [n]; entry of a rope's last vertex unused */);
RS_API int rs_batch_min_segment(rs_batch* b, float* out);
/* per-vertex arrays [n]; entries of pinned vertices (masses) or of each rope's last vertex
 * (EA, EI) are ignored */
RS_API int rs_batch_set_masses(rs_batch* b, const float* masses);
RS_API int rs_batch_set_stretch_stiffnesses(rs_batch* b, const float* ea);
RS_API int rs_batch_set_bend_stiffnesses(rs_batch* b, const float* ei);
RS_API int rs_batch_set_velocities(rs_batch* b, const float* vel /* host [n,3] */);
/* RopeSim::set_root (bindings.cpp:324-350): q (already unit) may be NULL */
RS_API int rs_batch_set_root(rs_batch* b, int rope, const float* pos3, const float* vel3, const float* q4);
RS_API int rs_batch_unpin_root(rs_batch* b, int rope);
RS_API int rs_batch_roots_pinned(rs_batch* b, int* pinned);

/* ---------------------------------------------------------------- stepping
 * One control frame = ONE persistent kernel launch over every substep.
 * step_program replaces RopeBatch::step_program (batch.cu:321-363): p0, v0, p1 [R,3], q0, q1
 * [R,4] or NULL; `on_host` = 1 when the pointers are host memory (copied in), else device.
 * step_legacy replaces RopeBatch::step (batch.cu:288-319): p, v [R,3], q [R,4] or NULL.
 * step_free replaces RopeBatch::step_free (batch.cu:388-398).
 * advance replaces RopeSim::advance / Sim::advance (bindings.cpp:274-295, step.cpp:37-57):
 * substeps = 0 runs the float ceil(dt / max_h) substeps. */
RS_API int rs_batch_step_program(rs_batch* b, const float* p0, const float* v0, const float* p1, const float* q0,
                          const float* q1, float dt, int substeps, int on_host);
RS_API int rs_batch_step_legacy(rs_batch* b, const float* p, const float* v, const float* q, float dt, int substeps,
                         int on_host);
RS_API int rs_batch_step_free(rs_batch* b, float dt, int substeps);
/* rs_batch_step_program with device inputs (on_host = 0) that allocates no device memory. No
 * counterpart in the reference. For callers that cannot call cudaMalloc once the simulation is
 * running: hosts that reserve all device memory up front for their own allocator (physics or
 * rendering engines that embed this library, ML runtimes that preallocate the GPU), real-time
 * control loops whose memory is fixed at start-up, and runtimes that forbid allocation after
 * initialisation. The regular step needs no new allocation per frame either, but its
 * rope-rope candidate lists live in a buffer the handle allocates when contact is enabled, and
 * autotuning or a pending host edit can reallocate; this entry point instead keeps the lists in
 * the library's static device array (128 x 8192 ints = 4 MiB, held by every GPU that loads the
 * library until exit) and refuses, with RS_EINVAL and a message, batches of more than 8192
 * vertices, pending host edits, contact groups larger than one CTA, and the plain engine. The
 * array's device address is looked up on the first call on each device (keep that first call
 * outside any stream capture). All such calls share the array: calls that overlap on the GPU
 * race. Results equal rs_batch_step_program's, bit for bit. The handle's own candidate buffer
 * is still allocated when rope contact is enabled (rs_batch_set_rope_contact, at set-up), so
 * the static array saves no memory: what it removes is any allocation while stepping. With
 * rs_batch_set_timing on, rs_batch_last_frame_ms reports this call's frame kernel too. */
RS_API int rs_batch_step_program_static_scratch(rs_batch* b, const float* p0, const float* v0, const float* p1,
                                                const float* q0, const float* q1, float dt, int substeps);
RS_API int rs_batch_advance(rs_batch* b, float dt, int substeps);
/* RopeBatch::reset_envs (batch.cu:400-413): host ids[count] (rope indices) */
RS_API int rs_batch_reset_ropes(rs_batch* b, const int* ids, int count);
/* RopeSim::reset (bindings.cpp:303-316) */
RS_API int rs_batch_reset_all(rs_batch* b);
/* RopeBatch::gather (batch.cu:420-425) */
RS_API int rs_batch_gather(rs_batch* b);
/* Device views [n,3], [n,3], [n,4] (caller order), refreshed by every step/reset/gather;
 * stable for the handle's life (RopeBatch::positions_ptr etc., batch.h:79-81). */
RS_API int rs_batch_views(rs_batch* b, float** pos, float** vel, float** quat);
/* Solver status (Sim::lastErrorCode / lastWarningCode, bindings.cpp:578-579) and a sticky
 * flag raised when a frame produced a non-finite position. */
RS_API int rs_batch_status(rs_batch* b, int* last_error, int* last_warning, int* nonfinite);
/* The checked build (libropesim_b200_checked.so, compiled with -DROPESIM_CHECKED) tests every
 * neighbour, candidate, pose-cache, lattice, caller and group index its frame and adjoint kernels
 * use and records the first failed check (code: 1 bin range, 2 next-vertex read, 3 previous-vertex
 * read, 4 caller / rope index, 5 contact-group range, 6 candidate segment, 7 pose-cache slot or
 * mesh bit, 8 lattice node, 9 lattice block bound; 0 = none) instead of trapping; the access is
 * skipped or kept in range. *code: that record (sticky; always 0 in the regular build);
 * *checked: 1 in the checked build. No counterpart in the reference (a stand-in for running the
 * kernels under a memory checker). */
RS_API int rs_batch_bounds_check(rs_batch* b, int* code, int* checked);
/* CUDA stream the handle's device work runs on. */
RS_API int rs_batch_stream(rs_batch* b, void** stream);
/* Device time of the last frame kernel in ms (after rs_batch_set_timing(b, 1)). */
RS_API int rs_batch_set_timing(rs_batch* b, int on);
RS_API int rs_batch_last_frame_ms(rs_batch* b, double* ms);

/* ---------------------------------------------------------------- surface contact
 * set_contact / set_planes replace write_contact / write_planes (bindings.cpp:51-80): rows are
 * [count <= 8, 4] = (n, w) half-spaces n.x >= w, normalised here. */
RS_API int rs_batch_set_contact(rs_batch* b, float radius, float mu_s, float mu_k, float v_slip, float kappa);
RS_API int rs_batch_get_contact(rs_batch* b, float* radius, float* mu_s, float* mu_k);
RS_API int rs_batch_set_planes(rs_batch* b, int count, const float* rows);
/* RopeBatch::set_rope_contact (batch.cu:367-385, bindings.cpp:939-950): YarnBall's rope-rope
 * model (log barrier at 2 radius + barrier, friction spring capped at mu N, step limit) on
 * candidates from a per-group brute-force detector; group_ropes consecutive ropes form one
 * contact group. Groups that fit one CTA (<= 1024 vertices) stay on the persistent kernel;
 * larger groups run on the plain engine. enabled = 0 switches it off. */
RS_API int rs_batch_set_rope_contact(rs_batch* b, int enabled, float radius, float barrier, float k_collision, float mu,
                                     float k_friction, float detection_scaler, int group_ropes);
/* SdfStore::add (sdf.cu:137-158): values host [nx,ny,nz], pose rows host [rows,3]/[rows,4]
 * (rows 1 or num_ropes). Returns the mesh index in *index. */
RS_API int rs_batch_add_mesh(rs_batch* b, const float* values, int nx, int ny, int nz, const float* origin3,
                      float spacing, float mu_s, float mu_k, const float* pos, const float* quat, int rows,
                      int* index);
RS_API int rs_batch_set_mesh_friction(rs_batch* b, int index, float mu_s, float mu_k);
/* SdfStore::set_targets / set_targets_host (sdf.cu:165-189): index >= 0 with rows 1 or
 * num_ropes, or index = -1 with [num_ropes, M] rows; tele [num_ropes] or NULL; tele_all;
 * on_device = 1 when pos/quat/tele are device memory, 3 when pos/quat are device memory and tele
 * is host memory (staged, as the reference stages host flags given with CUDA poses). */
RS_API int rs_batch_set_mesh_poses(rs_batch* b, int index, const float* pos, const float* quat, int rows,
                            const uint8_t* tele, int tele_all, int on_device);
RS_API int rs_batch_clear_meshes(rs_batch* b);
RS_API int rs_batch_num_meshes(rs_batch* b, int* count);
RS_API int rs_batch_enable_contact_forces(rs_batch* b, int on);
/* averaged over the last frame: forces [n,3] ON each vertex; wrenches [num_ropes, M, 6] BY the
 * rope ON each mesh (SdfStore::contact_forces / wrenches, sdf.cu:255-270) */
RS_API int rs_batch_contact_forces(rs_batch* b, float* out);
RS_API int rs_batch_mesh_wrenches(rs_batch* b, float* out);
/* device views [n,3] and [num_ropes, 64, 6] (contact_forces_view / mesh_wrenches_view) */
RS_API int rs_batch_contact_views(rs_batch* b, float** forces, float** wrenches);

/* ---------------------------------------------------------------- differentiable frames
 * No counterpart in the reference, which has no gradients. What is differentiated is the
 * deterministic substep (root program, inertial prediction, num_itr x (position step with
 * inertia, plane contact and friction, stretch, damping; frame step), velocity with linear and
 * quadratic drag), with plane, static SDF-mesh and rope-rope contact (barrier, damping,
 * friction, closest points, step limit); branches (contact active, friction regime, frame-step
 * signs, step-limit clips) are held where the forward pass took them. A frame during which a
 * mesh moves is refused (RS_EINVAL).
 *
 * State: pos / vel / lvel [n,3], q [n,4], caller order; lvel is the velocity at the last
 * substep's start (the next substep's initial guess extrapolates from it). Parameters: ea / ei
 * [n] per segment i -> i+1 (a rope's last vertex is ignored), mass [n] (pinned vertices are
 * ignored). on_device = 1 for device pointers; a NULL pointer leaves that part unchanged.
 * rs_batch_set_parameters works between any two frames (the reference's per-vertex setters
 * only before the first step). */
RS_API int rs_batch_set_state(rs_batch* b, const float* pos, const float* vel, const float* lvel, const float* q,
                              int on_device);
RS_API int rs_batch_get_state(rs_batch* b, float* pos, float* vel, float* lvel, float* q, int on_device);
RS_API int rs_batch_set_parameters(rs_batch* b, const float* ea, const float* ei, const float* mass, int on_device);
RS_API int rs_batch_get_parameters(rs_batch* b, float* ea, float* ei, float* mass, int on_device);
/* One frame reversed (all pointers device, caller order). Inputs: the frame-start state, the
 * frame's program rows (p0 = NULL: a step_free frame; q0 / q1 optional, not differentiated),
 * the adjoints of the frame-end state (NULL = zero). Outputs: the adjoints of the frame-start
 * state (required) and, where non-NULL, of ea / ei / mass [n] and of p0 / v0 / p1 [R,3].
 * dt / substeps are the frame's; last_h is RS_P_H read before the frame was stepped. The frame
 * is replayed from the given state (the handle's own state is left untouched), recording each
 * substep's start state in a device tape of 64 B per vertex-substep, then reversed; with
 * io->tape set (recorded by rs_batch_step_program_taped) the replay is skipped. */
typedef struct rs_backward_io {
    const float *pos, *vel, *lvel, *q;
    const float *p0, *v0, *p1, *q0, *q1;
    const float *g_pos, *g_vel, *g_lvel, *g_q;
    float *o_pos, *o_vel, *o_lvel, *o_q;
    float *o_ea, *o_ei, *o_mass;
    float *o_p0, *o_v0, *o_p1;
    const float* tape;  /* NULL = replay the frame; else this frame's recorded tape */
    const float *ea, *ei, *mass;  /* the frame's parameters (NULL = the handle's current ones) */
    const float* itape; /* the frame's iterate tape (rs_frame_io.itape) or NULL (recompute) */
} rs_backward_io;
RS_API int rs_batch_backward(rs_batch* b, const rs_backward_io* io, float dt, int substeps, float last_h);
/* The same, returning with the work queued on the handle's stream (no host synchronization). */
RS_API int rs_batch_backward_async(rs_batch* b, const rs_backward_io* io, float dt, int substeps, float last_h);
/* One differentiable frame in one call (device pointers, caller order): loads the frame-start
 * state and the parameters (NULL = keep), steps with the program rows p0 / v0 / p1 [R,3] (all
 * three NULL: a free frame, as rs_batch_step_free), writes the end state to out_* and, when
 * tape != NULL (16 * substeps * n floats), the substep tape for rs_batch_backward. With itape
 * != NULL as well (12 * num_itr * substeps * n floats: every iterate d^k, q^k of every substep and
 * each frame step's blend rotor and sign tests) the backward reads the iterates instead of
 * recomputing them; without rope-rope contact and on the persistent engine only (elsewhere it is
 * ignored and the backward recomputes). *last_h receives the frame's lastH (RS_P_H before the
 * frame). Queued on the handle's stream without host synchronization. */
typedef struct rs_frame_io {
    const float *pos, *vel, *lvel, *q;
    const float *ea, *ei, *mass;
    const float *p0, *v0, *p1;
    float *out_pos, *out_vel, *out_lvel, *out_q;
    float* tape;
    float* itape;
} rs_frame_io;
RS_API int rs_batch_frame_forward(rs_batch* b, const rs_frame_io* io, float dt, int substeps, float* last_h);
/* rs_batch_step_program that also records the frame's substep tape for rs_batch_backward:
 * tape = device buffer of 16 * substeps * n floats (the state after each substep's root
 * program, caller order), so that the backward need not replay the frame. */
RS_API int rs_batch_step_program_taped(rs_batch* b, const float* p0, const float* v0, const float* p1,
                                       const float* q0, const float* q1, float dt, int substeps, float* tape);

/* ---------------------------------------------------------------- mesh baking
 * Replaces ropesim.sdf.bake_mesh's Warp kernel (ropesim/sdf.py:96-167): the signed distance of
 * every node origin + (i, j, k) * spacing (float32 of the float64 sum, C order [nx, ny, nz]) to
 * a triangle mesh (host vertices [num_vertices, 3], host triangles [num_triangles, 3], any
 * winding): exact closest-point distance, negative where the generalized winding number's
 * magnitude exceeds 1/2 (inside a closed mesh). thickness > 0 bakes the two-sided shell
 * |distance| - thickness / 2 instead (open meshes); round > 0 subtracts round. The lattice box
 * and the closedness check are the caller's (the Python bake_mesh does both as the reference).
 * out: host memory (out_on_device = 0; the call returns when it is filled) or device memory
 * (out_on_device = 1; queued on `stream`, NULL = the legacy default stream). counters: NULL or
 * host [4] receiving the point-triangle distances, line-triangle crossing tests and solid
 * angles evaluated and the kernels' device time in nanoseconds, the host preparation (triangle
 * sort and upload) excluded; the call then synchronizes. Zero-area triangles are dropped. RS_EINVAL on
 * bad sizes or indices, or more than 7000 nodes along z. */
RS_API int rs_sdf_bake(const float* vertices, int num_vertices, const int* triangles, int num_triangles,
                       const float* origin3, double spacing, int nx, int ny, int nz, float thickness, float round,
                       float* out, int out_on_device, void* stream, unsigned long long* counters);

/* ---------------------------------------------------------------- measurement
 * Measured FP32 FMA throughput of the current device in TFLOP/s (2 FLOP per FMA), from a
 * kernel of independent FMA chains (no counterpart in the reference; bench.py uses it as the
 * roofline peak of the FP32-bound frame kernel). */
RS_API int rs_probe_fp32_peak(double* tflops, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* ROPESIM_B200_H */
