// rs_kernels.h -- host-side launchers of the kernels in rs_frame.cu, rs_plain.cu and rs_adjoint.cu.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "rs_types.h"

namespace rs {

// One persistent launch that runs every substep of one control frame for every bin.
cudaError_t launch_frame(const FrameArgs& a, int block, int num_bins, cudaStream_t s);
// Everything launch_frame does on the host before its launch (load the kernel, set its shared
// memory limit, count its resident CTAs), without launching: run before a timed launch.
cudaError_t prepare_frame(const FrameArgs& a, int block);
// Device state -> caller-order views.
cudaError_t launch_gather(const FrameArgs& a, int n, cudaStream_t s);
// Restore construction state of device vertex ranges (x = start, y = count).
cudaError_t launch_reset(float4* pos, float4* vel, float4* lvel, float4* q, const float4* init_pos, const float4* init_q,
                         const int2* ranges, int count, int maxv, cudaStream_t s);
// Mesh pose machine.
cudaError_t launch_scatter_targets(Pose7* tgt, uint8_t* tele, int index, const float* pos, const float* quat, int rows,
                                   int M, const uint8_t* tele_flags, int tele_all, int N, cudaStream_t s);
cudaError_t launch_stage_motion(Pose7* cur, const Pose7* tgt, uint8_t* tele, Motion* motion, int total, cudaStream_t s);
cudaError_t launch_commit(Pose7* cur, const Pose7* tgt, uint8_t* tele, Pose* poses, const float* boxes, int num_sdf,
                          int only, int N, cudaStream_t s);
cudaError_t launch_scale(float* x, int n, float k, cudaStream_t s);
// Plain (per-substep-launch) engine: `pa` is the frame's FrameArgs in device memory.
cudaError_t plain_record_inner(const FrameArgs* pa, const PlainBufs& b, int n, int iters, int surf, bool rope,
                               cudaStream_t s);
cudaError_t plain_launch_pre(const FrameArgs* pa, const PlainBufs& b, int n, int nropes, int envs, int num_sdf, bool moving,
                             int root_mode, bool rope, int s, const RopeGrid* grid, cudaStream_t st);
// Rope-rope detection through a uniform grid (rs_ropegrid.cu), the brute force's candidate lists,
// for contact groups larger than one CTA: `pos` the substep-start positions (device order).
int rope_grid_buckets(int n);
size_t rope_grid_scan_bytes(int T);
cudaError_t rope_grid_detect(const FrameArgs* pa, const float4* pos, const RopeGrid& g, int n, bool flag, cudaStream_t st);
cudaError_t plain_launch_finish(const FrameArgs* pa, const PlainBufs& b, int n, cudaStream_t st);
// Device address of the library's static rope-rope candidate array on the current device and
// its capacity in vertices (looked up once per device, then cached; no allocation).
cudaError_t static_scratch_cols(int** ptr, int* max_verts);
// Differentiable frames (rs_adjoint.cu): one frame's reverse sweep from the tape that a frame
// launch with a.tape set wrote; shared memory it needs per CTA.
cudaError_t launch_adjoint(const FrameArgs& a, const AdjArgs& g, int block, int num_bins, cudaStream_t s);
size_t adjoint_smem_bytes(int block, int iters, bool rope);
// The same reverse sweep as per-vertex launches over HBM arrays (rs_adjoint_plain.cu), for
// contact groups larger than one CTA and the plain engine: `pa` is the frame's FrameArgs in
// device memory; its arrays are carved from one float4 buffer of adjoint_plain_words(n, iters).
size_t adjoint_plain_words(int n, int iters);
PlainAdjBufs adjoint_plain_carve(float4* base, int n, int iters);
cudaError_t launch_adjoint_plain(const FrameArgs* pa, const AdjArgs& g, const PlainAdjBufs& b, int n, int iters,
                                 int substeps, int surf, bool rope, const RopeGrid* grid, cudaStream_t st);
// Caller-order state <-> device order (the .w constants of cst_* are kept).
cudaError_t launch_state_in(const int4* topo, const float* pos, const float* vel, const float* lvel, const float* q,
                            const float4* cst_pos, const float4* cst_vel, const float4* cst_lvel, float4* o_pos,
                            float4* o_vel, float4* o_lvel, float4* o_q, int n, cudaStream_t s);
cudaError_t launch_state_out(const int4* topo, const float4* pos, const float4* vel, const float4* lvel, const float4* q,
                             float* o_pos, float* o_vel, float* o_lvel, float* o_q, int n, cudaStream_t s);
// Per-vertex EA / EI / mass in caller order -> device constants, and back.
cudaError_t launch_params_in(const int4* topo, const float* ea, const float* ei, const float* mass, float4* pos,
                             const float4* vel, float4* lvel, float4* qrest, const float4* qdir, int n, cudaStream_t s);
cudaError_t launch_params_out(const int4* topo, const float4* pos, const float4* vel, const float4* lvel,
                              const float4* qrest, float* ea, float* ei, float* mass, int n, cudaStream_t s);
// FP32 FMA throughput probe (16 * 8 FMAs per thread per iteration).
cudaError_t launch_fp32_probe(float* out, int blocks, int threads, int iters, cudaStream_t s);
// Signed-distance lattice of a triangle mesh (rs_sdfbake.cu): host vertices [nv,3] and
// triangles [nt,3]; `out` [nx,ny,nz] host (synchronous) or device (queued on s); counters NULL
// or [4] host (distance evaluations, crossing tests, solid angles, kernel nanoseconds). On a validation failure
// *err is set and cudaErrorInvalidValue returned.
cudaError_t sdf_bake(const float* verts, int nv, const int* tris, int nt, const float* origin, double spacing, int nx, int ny,
                     int nz, float thickness, float round, float* out, bool out_on_device, unsigned long long* counters,
                     cudaStream_t s, std::string* err);

}  // namespace rs
