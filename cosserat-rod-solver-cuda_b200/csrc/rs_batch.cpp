// rs_batch.cpp -- host driver: setup, packing, staging, mesh pose machine, frame launch.
#include "rs_batch.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>

#include "rs_kernels.h"

namespace rs {

namespace {

// Single-precision rotor helpers for the host setup. The setup follows YarnBall.cu:112-259
// operation by operation (same order, IEEE float, no contraction) so that initial frames and
// rest rotations are the reference's.
V4 qmul(const V4& a, const V4& b) {
    // (a.w b.v + b.w a.v + a.v x b.v, a.w b.w - a.v . b.v), Rotor.h:185-188
    const float cx = a.y * b.z - a.z * b.y, cy = a.z * b.x - a.x * b.z, cz = a.x * b.y - a.y * b.x;
    V4 r;
    r.x = (a.w * b.x + b.w * a.x) + cx;
    r.y = (a.w * b.y + b.w * a.y) + cy;
    r.z = (a.w * b.z + b.w * a.z) + cz;
    r.w = a.w * b.w - ((a.x * b.x + a.y * b.y) + a.z * b.z);
    return r;
}
V4 qconj(const V4& a) { return V4{-a.x, -a.y, -a.z, a.w}; }
float dot4(const V4& a, const V4& b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + a.w * b.w); }
V4 scale4(const V4& a, float s) { return V4{a.x * s, a.y * s, a.z * s, a.w * s}; }
V4 normalize4(const V4& a) { return scale4(a, 1.f / std::sqrt(dot4(a, a))); }

int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

void Batch::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw cuda_error(std::string(what) + ": " + cudaGetErrorString(e));
}

Batch::Batch(int num_ropes, const int* rope_verts, const float* positions, const uint8_t* pinned, float density,
             float k_stretch, float k_bend, float max_h_in, int num_itr_in, bool fix_root_orientation,
             bool straight_rest, float dead_radius, float dead_barrier) {
    if (num_ropes < 1) throw std::invalid_argument("num_ropes must be >= 1");
    R_ = num_ropes;
    ustart_.assign(R_ + 1, 0);
    for (int r = 0; r < R_; r++) {
        if (rope_verts[r] < 3) throw std::invalid_argument("every rope needs >= 3 vertices");
        if (rope_verts[r] > 1024) throw std::invalid_argument("ropes longer than 1024 vertices are not supported");
        ustart_[r + 1] = ustart_[r] + rope_verts[r];
        if (rope_verts[r] != rope_verts[0]) uniform_ = false;
    }
    n_ = ustart_[R_];
    im_.assign(n_, 1.f); lr_.assign(n_, 1.f); ks_.assign(n_, 100.f); fl_.assign(n_, F_NEXT);
    qrest_.assign(n_, V4{0.f, 0.f, 0.f, 5.f});
    pos_.assign(n_, V4{0, 0, 0, 0}); vel_.assign(n_, V4{0, 0, 0, 0}); lvel_.assign(n_, V4{0, 0, 0, 0});
    q_.assign(n_, V4{0, 0, 0, 1});
    for (int i = 0; i < n_; i++) pos_[i] = V4{positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0.f};
    fl_[n_ - 1] = 0;
    // RopeBatch ctor, batch.cu:344-361
    for (int r = 0; r < R_; r++) {
        fl_[ustart_[r + 1] - 1] = 0;
        for (int i = ustart_[r]; i < ustart_[r + 1]; i++)
            if (pinned ? pinned[i] != 0 : i == ustart_[r]) im_[i] = 0.f;
        if (fix_root_orientation) fl_[ustart_[r]] |= F_FIX_ORIENT;
    }
    configure(density);
    rc_radius_ = dead_radius;
    rc_barrier_ = dead_barrier;
    // dead collision radii gate the segment-length check of uploadMeta (YarnBall.cu:268)
    if (2.f * min_seg_ < 2.f * dead_radius + dead_barrier)
        throw std::invalid_argument("Use thinner yarn or use longer segments (2 * min segment >= 2 * radius + barrier)");
    if (straight_rest)
        for (int r = 0; r < R_; r++)
            for (int i = ustart_[r]; i + 1 < ustart_[r + 1]; i++) qrest_[i] = V4{0.f, 0.f, 0.f, 1.f};
    for (int i = 0; i < n_; i++) ks_[i] = k_stretch * lr_[i];       // setKStretch
    const float kb4 = k_bend * 4.f;                                   // setKBend
    qdir_.resize(n_);
    for (int i = 0; i < n_; i++) {
        qdir_[i] = normalize4(qrest_[i]);  // kept: set_parameters scales these directions
        qrest_[i] = scale4(qdir_[i], kb4 / lr_[i]);
    }
    for (int r = 0; r < R_; r++) fl_[ustart_[r]] |= F_ROOT;
    max_h = max_h_in;
    h_ = max_h_in;   // seed lastH like a fresh sim (bindings.cpp:249-253)
    num_itr = num_itr_in;
    init_pos_ = pos_;
    init_q_ = q_;

    check(cudaStreamCreate(&stream_), "cudaStreamCreate");
    check(cudaEventCreate(&ev0_), "cudaEventCreate");
    check(cudaEventCreate(&ev1_), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&ev_cost_, cudaEventDisableTiming), "cudaEventCreate");
    host_dyn_valid_ = true;
    device_valid_ = false;
    layout_valid_ = false;
    ensure_device();
    gather();   // views are valid before the first step (batch.cu:411)
    check(cudaStreamSynchronize(stream_), "construct");
}

Batch::~Batch() {
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& g : grids_) {
        cudaFree(const_cast<float*>(g.v));
        cudaFree(const_cast<float*>(g.bmin));
    }
    void* bufs[] = {d_bins_, d_ropes_, d_topo_, d_pos_, d_vel_, d_lvel_, d_q_, d_qrest_, d_qdir_, d_init_pos_, d_init_q_,
                    d_out_pos_, d_out_vel_, d_out_q_, d_prog_, d_status_, d_ranges_, d_boxes_, d_cur_, d_tgt_,
                    d_tele_, d_motion_, d_poses_, d_stage_, d_stage_tele_, d_force_, d_wrench_, d_queue_, d_order_,
                    d_bin_cost_};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (pl_graph_) cudaGraphExecDestroy(pl_graph_);
    void* pbufs[] = {pl_.dx, pl_.dxn, pl_.y, pl_.qprev, pl_.lpos, pl_.facc, pl_.cand, pl_.spose, d_pl_args_,
                     d_grp_, d_cols_, d_ncols_, d_maxstep_, d_pad_, gs_pos_, gs_vel_, gs_lvel_, gs_q_, gs_buf_, d_tape_,
                     d_padj_, d_adj_args_, grid_mem_};
    for (void* p : pbufs)
        if (p) cudaFree(p);
    if (h_pl_args_) cudaFreeHost(h_pl_args_);
    if (h_adj_args_) cudaFreeHost(h_adj_args_);
    if (h_prog_) cudaFreeHost(h_prog_);
    if (h_status_) cudaFreeHost(h_status_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev_cost_) cudaEventDestroy(ev_cost_);
    if (h_bin_cost_) cudaFreeHost(h_bin_cost_);
    if (h_order_) cudaFreeHost(h_order_);
    if (stream_) cudaStreamDestroy(stream_);
}

// Sim::configure, YarnBall.cu:112-182. Frames are transported along the whole caller-order
// array, so each rope's initial frames continue from the previous rope's last frame.
void Batch::configure(float density) {
    max_seg_ = 0.f;
    min_seg_ = std::numeric_limits<float>::max();
    V4 lastQ{0.f, 0.f, 0.f, 1.f};
    for (int i = 0; i < n_; i++) {
        if (i < n_ - 1) {
            const bool hasNext = fl_[i] & F_NEXT;
            fl_[i + 1] = hasNext ? (fl_[i + 1] | F_PREV) : (fl_[i + 1] & ~F_PREV);
            const bool hasNextNext = hasNext && (fl_[i + 1] & F_NEXT);
            fl_[i] = hasNextNext ? (fl_[i] | F_NEXT_ORIENT) : (fl_[i] & ~F_NEXT_ORIENT);
            if (!hasNext) fl_[i] |= F_FIX_ORIENT;
        }
        if (!(fl_[i] & F_PREV) && !(fl_[i] & F_NEXT))
            throw std::invalid_argument("Dangling segment. Yarns must be atleast 2 segments long");
        lr_[i] = 1.f / (float)n_;
        float mass = 0.f;
        if (fl_[i] & F_PREV) mass += lr_[i - 1];
        if (fl_[i] & F_NEXT) {
            const float sx = pos_[i + 1].x - pos_[i].x, sy = pos_[i + 1].y - pos_[i].y, sz = pos_[i + 1].z - pos_[i].z;
            const float d2 = (sx * sx + sy * sy) + sz * sz;
            lr_[i] = std::sqrt(d2);
            if (lr_[i] == 0.f || !std::isfinite(lr_[i])) throw std::invalid_argument("0 length segment");
            const float inv = 1.f / std::sqrt(d2);
            const float dx = sx * inv, dy = sy * inv, dz = sz * inv;
            V4 qq;
            if (dx < -0.999999f) {
                qq = V4{0.f, 0.f, 1.f, 0.f};
            } else {  // Rotor::fromTo(e1, d), Rotor.h:57-64
                float hx = (1.f + dx) * 0.5f, hy = (0.f + dy) * 0.5f, hz = (0.f + dz) * 0.5f;
                const float l = (hx * hx + hy * hy) + hz * hz;
                if (l > 0.f) {
                    const float s = 1.f / std::sqrt(l);
                    hx *= s; hy *= s; hz *= s;
                } else {
                    hx = 0.f; hy = 1.f; hz = 0.f;
                }
                // cross(e1, h), dot(e1, h)
                qq = V4{0.f * hz - 0.f * hy, 0.f * hx - 1.f * hz, 1.f * hy - 0.f * hx, (1.f * hx + 0.f * hy) + 0.f * hz};
            }
            V4 t = qmul(qconj(qq), lastQ);
            const V4 tw{t.x, 0.f, 0.f, t.w};
            t = (dot4(tw, tw) > 1e-12f) ? normalize4(tw) : V4{0.f, 0.f, 0.f, 1.f};
            lastQ = qmul(qq, t);
            mass += lr_[i];
            max_seg_ = std::max(max_seg_, lr_[i]);
            min_seg_ = std::min(min_seg_, lr_[i]);
        }
        q_[i] = lastQ;
        mass *= 0.5f * density;
        im_[i] = (mass != 0.f) ? im_[i] * (1.f / mass) : 0.f;
    }
    for (int i = 0; i < n_ - 1; i++) qrest_[i] = scale4(qmul(qconj(q_[i]), q_[i + 1]), std::sqrt(dot4(qrest_[i], qrest_[i])));
}

bool Batch::roots_pinned() const {
    for (int r = 0; r < R_; r++)
        if (im_[ustart_[r]] != 0.f) return false;
    return true;
}

int Batch::pose_cache_entries() const { return std::max(1, max_rcount_ * (int)grids_.size()); }

// Whole ropes into bins of `block_` threads: first-fit decreasing by length; a bin also
// holds at most max_ropes_per_bin_ ropes (bounded by the per-CTA mesh pose cache).
// Whole ropes into bins of `block_` threads: first-fit decreasing by size over *units* -- single
// ropes, or whole rope-rope contact groups (group_ropes consecutive ropes, kept in caller order
// so that detection scans candidates in the reference's order). A bin also holds at most
// max_ropes_per_bin_ ropes (bounded by the per-CTA mesh pose cache). A contact group larger
// than the largest CTA cannot be CTA-resident: the layout then keeps caller order and frames run
// on the plain engine.
void Batch::pack() {
    std::vector<std::vector<int>> units;
    const int G = rope_contact_ ? std::max(1, group_ropes_) : 1;
    for (int r0 = 0; r0 < R_; r0 += G) {
        std::vector<int> u;
        for (int r = r0; r < std::min(R_, r0 + G); r++) u.push_back(r);
        units.push_back(u);
    }
    auto usize = [&](const std::vector<int>& u) {
        int v = 0;
        for (int r : u) v += rope_verts(r);
        return v;
    };
    int maxU = 0;
    for (auto& u : units) maxU = std::max(maxU, usize(u));
    max_unit_verts_ = maxU;
    oversize_ = maxU > 1024;
    int blk = block_override ? block_override : tune_block_;
    if (blk == 0) {
        blk = std::max(64, next_pow2(std::min(maxU, 1024)));
        if (blk < 256 && (long long)n_ > 148LL * blk) blk = 256;
    }
    if (!oversize_ && blk < maxU) blk = next_pow2(maxU);
    block_ = std::min(blk, 1024);
    const int M = (int)grids_.size();
    int cap = max_ropes_per_bin_;
    if (M > 0) cap = std::min(cap, std::max(1, (96 * 1024) / (2 * M * (int)(sizeof(Pose) + 2 * sizeof(float4)))));
    std::vector<int> order(units.size());
    std::iota(order.begin(), order.end(), 0);
    if (!oversize_)
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return usize(units[a]) > usize(units[b]); });
    struct Open { int used, rc; std::vector<int> ropes; };
    std::vector<Open> open;
    int first_open = 0;
    for (int ui : order) {
        const int L = usize(units[ui]);
        const int nr = (int)units[ui].size();
        int b = -1;
        if (!oversize_)
            for (int k = first_open; k < (int)open.size(); k++)
                if (open[k].used + L <= block_ && open[k].rc + nr <= std::max(cap, nr)) { b = k; break; }
        if (b < 0) { open.push_back(Open{0, 0, {}}); b = (int)open.size() - 1; }
        open[b].used += L;
        open[b].rc += nr;
        for (int r : units[ui]) open[b].ropes.push_back(r);
        while (first_open < (int)open.size() && (open[first_open].used + 3 > block_ || open[first_open].rc >= cap)) first_open++;
    }
    bins_.clear();
    dropes_.clear();
    u2d_.assign(n_, 0);
    int dv = 0;
    max_rcount_ = 1;
    for (auto& o : open) {
        Bin b{dv, 0, (int)dropes_.size(), (int)o.ropes.size()};
        for (int r : o.ropes) {
            Rope rp{dv, rope_verts(r), ustart_[r], r};
            for (int i = 0; i < rp.count; i++) u2d_[rp.ustart + i] = dv + i;
            dv += rp.count;
            dropes_.push_back(rp);
        }
        b.vcount = dv - b.vstart;
        bins_.push_back(b);
        max_rcount_ = std::max(max_rcount_, b.rcount);
    }
    // contact-group and rope ranges per device vertex (device order)
    grp_.assign(n_, int4{0, 0, 0, 0});
    for (auto& u : units) {
        const int gs = u2d_[ustart_[u.front()]];
        const int ge = u2d_[ustart_[u.back()]] + rope_verts(u.back());
        for (int r : u) {
            const int rs0 = u2d_[ustart_[r]];
            for (int i = 0; i < rope_verts(r); i++) grp_[rs0 + i] = int4{gs, ge, rs0, rs0 + rope_verts(r)};
        }
    }
}

void Batch::alloc_device() {
    auto alloc = [&](void** p, size_t bytes, const char* what) {
        if (*p) cudaFree(*p);
        *p = nullptr;
        check(cudaMalloc(p, bytes), what);
    };
    alloc((void**)&d_bins_, sizeof(Bin) * bins_.size(), "cudaMalloc(bins)");
    alloc((void**)&d_order_, sizeof(int) * bins_.size(), "cudaMalloc(bin order)");
    alloc((void**)&d_bin_cost_, sizeof(float) * bins_.size(), "cudaMalloc(bin times)");
    if (!d_queue_) alloc((void**)&d_queue_, sizeof(int), "cudaMalloc(work queue)");
    if (h_bin_cost_) cudaFreeHost(h_bin_cost_);
    if (h_order_) cudaFreeHost(h_order_);
    h_bin_cost_ = nullptr;
    h_order_ = nullptr;
    check(cudaMallocHost((void**)&h_bin_cost_, sizeof(float) * bins_.size()), "cudaMallocHost(bin times)");
    check(cudaMallocHost((void**)&h_order_, sizeof(int) * bins_.size()), "cudaMallocHost(bin order)");
    alloc((void**)&d_ropes_, sizeof(Rope) * dropes_.size(), "cudaMalloc(ropes)");
    if (!d_pos_) {
        const size_t n4 = sizeof(float4) * n_;
        alloc((void**)&d_topo_, sizeof(int4) * n_, "cudaMalloc(topo)");
        alloc((void**)&d_pos_, n4, "cudaMalloc(pos)");
        alloc((void**)&d_vel_, n4, "cudaMalloc(vel)");
        alloc((void**)&d_lvel_, n4, "cudaMalloc(lvel)");
        alloc((void**)&d_q_, n4, "cudaMalloc(q)");
        alloc((void**)&d_qrest_, n4, "cudaMalloc(qrest)");
        alloc((void**)&d_qdir_, n4, "cudaMalloc(qrest directions)");
        alloc((void**)&d_init_pos_, n4, "cudaMalloc(init pos)");
        alloc((void**)&d_init_q_, n4, "cudaMalloc(init q)");
        alloc((void**)&d_out_pos_, sizeof(float) * 3 * n_, "cudaMalloc(view pos)");
        alloc((void**)&d_out_vel_, sizeof(float) * 3 * n_, "cudaMalloc(view vel)");
        alloc((void**)&d_out_q_, sizeof(float) * 4 * n_, "cudaMalloc(view quat)");
        alloc((void**)&d_prog_, sizeof(float) * 17 * R_, "cudaMalloc(program)");
        alloc((void**)&d_status_, sizeof(int) * 4, "cudaMalloc(status)");
        alloc((void**)&d_ranges_, sizeof(int2) * R_, "cudaMalloc(reset ranges)");
        check(cudaMemset(d_status_, 0, sizeof(int) * 4), "memset(status)");
        check(cudaMemset(d_prog_, 0, sizeof(float) * 17 * R_), "memset(program)");
        check(cudaMallocHost((void**)&h_prog_, sizeof(float) * 17 * R_), "cudaMallocHost(program)");
        check(cudaMallocHost((void**)&h_status_, sizeof(int) * 4), "cudaMallocHost(status)");
        const size_t slots = (size_t)R_ * kMaxSdf;
        alloc((void**)&d_boxes_, sizeof(float) * 6 * kMaxSdf, "cudaMalloc(sdf boxes)");
        alloc((void**)&d_cur_, sizeof(Pose7) * slots, "cudaMalloc(sdf cur)");
        alloc((void**)&d_tgt_, sizeof(Pose7) * slots, "cudaMalloc(sdf tgt)");
        alloc((void**)&d_tele_, slots, "cudaMalloc(sdf tele)");
        alloc((void**)&d_motion_, sizeof(Motion) * slots, "cudaMalloc(sdf motion)");
        alloc((void**)&d_poses_, sizeof(Pose) * slots, "cudaMalloc(sdf poses)");
        alloc((void**)&d_stage_, sizeof(float) * 7 * slots, "cudaMalloc(sdf stage)");
        alloc((void**)&d_stage_tele_, R_, "cudaMalloc(sdf stage flags)");
        std::vector<Pose7> ident(slots, Pose7{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f});
        check(cudaMemcpy(d_cur_, ident.data(), sizeof(Pose7) * slots, cudaMemcpyHostToDevice), "upload(sdf cur)");
        check(cudaMemcpy(d_tgt_, ident.data(), sizeof(Pose7) * slots, cudaMemcpyHostToDevice), "upload(sdf tgt)");
        check(cudaMemset(d_tele_, 0, slots), "memset(sdf tele)");
        check(cudaMemset(d_poses_, 0, sizeof(Pose) * slots), "memset(sdf poses)");
        check(cudaMemset(d_motion_, 0, sizeof(Motion) * slots), "memset(sdf motion)");
        check(cudaMemset(d_boxes_, 0, sizeof(float) * 6 * kMaxSdf), "memset(sdf boxes)");
    }
}

void Batch::ensure_device() {
    if (!layout_valid_) {
        ensure_host();
        pack();
        alloc_device();
        std::vector<int4> topo(n_);
        std::vector<float4> ip(n_), iq(n_);
        for (const Bin& b : bins_)
            for (int r = b.rstart; r < b.rstart + b.rcount; r++) {
                const Rope& rp = dropes_[r];
                for (int i = 0; i < rp.count; i++) {
                    const int u = rp.ustart + i, d = rp.dstart + i;
                    topo[d] = make_int4((int)fl_[u], r - b.rstart, u, rp.user);
                    ip[d] = make_float4(init_pos_[u].x, init_pos_[u].y, init_pos_[u].z, 0.f);
                    iq[d] = make_float4(init_q_[u].x, init_q_[u].y, init_q_[u].z, init_q_[u].w);
                }
            }
        check(cudaMemcpy(d_bins_, bins_.data(), sizeof(Bin) * bins_.size(), cudaMemcpyHostToDevice), "upload(bins)");
        for (size_t i = 0; i < bins_.size(); i++) h_order_[i] = (int)i;  // first frame: packing order
        check(cudaMemcpy(d_order_, h_order_, sizeof(int) * bins_.size(), cudaMemcpyHostToDevice), "upload(bin order)");
        costs_inflight_ = false;
        check(cudaMemcpy(d_ropes_, dropes_.data(), sizeof(Rope) * dropes_.size(), cudaMemcpyHostToDevice), "upload(ropes)");
        check(cudaMemcpy(d_topo_, topo.data(), sizeof(int4) * n_, cudaMemcpyHostToDevice), "upload(topo)");
        check(cudaMemcpy(d_init_pos_, ip.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(init pos)");
        check(cudaMemcpy(d_init_q_, iq.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(init q)");
        if (!d_grp_) check(cudaMalloc(&d_grp_, sizeof(int4) * n_), "cudaMalloc(groups)");
        check(cudaMemcpy(d_grp_, grp_.data(), sizeof(int4) * n_, cudaMemcpyHostToDevice), "upload(groups)");
        layout_valid_ = true;
        device_valid_ = false;
    }
    if (!device_valid_) {
        std::vector<float4> P(n_), Vv(n_), L(n_), Q(n_), QR(n_), QD(n_);
        std::vector<int4> topo(n_);
        for (int u = 0; u < n_; u++) {
            const int d = u2d_[u];
            P[d] = make_float4(pos_[u].x, pos_[u].y, pos_[u].z, im_[u]);
            Vv[d] = make_float4(vel_[u].x, vel_[u].y, vel_[u].z, lr_[u]);
            L[d] = make_float4(lvel_[u].x, lvel_[u].y, lvel_[u].z, ks_[u]);
            Q[d] = make_float4(q_[u].x, q_[u].y, q_[u].z, q_[u].w);
            QR[d] = make_float4(qrest_[u].x, qrest_[u].y, qrest_[u].z, qrest_[u].w);
            QD[d] = make_float4(qdir_[u].x, qdir_[u].y, qdir_[u].z, qdir_[u].w);
        }
        for (const Bin& b : bins_)
            for (int r = b.rstart; r < b.rstart + b.rcount; r++) {
                const Rope& rp = dropes_[r];
                for (int i = 0; i < rp.count; i++) topo[rp.dstart + i] = make_int4((int)fl_[rp.ustart + i], r - b.rstart, rp.ustart + i, rp.user);
            }
        check(cudaMemcpy(d_topo_, topo.data(), sizeof(int4) * n_, cudaMemcpyHostToDevice), "upload(topo)");
        check(cudaMemcpy(d_pos_, P.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(pos)");
        check(cudaMemcpy(d_vel_, Vv.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(vel)");
        check(cudaMemcpy(d_lvel_, L.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(lvel)");
        check(cudaMemcpy(d_q_, Q.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(q)");
        check(cudaMemcpy(d_qrest_, QR.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(qrest)");
        check(cudaMemcpy(d_qdir_, QD.data(), sizeof(float4) * n_, cudaMemcpyHostToDevice), "upload(qrest directions)");
        device_valid_ = true;
    }
}

void Batch::ensure_host() {
    if (host_dyn_valid_ && !host_const_stale_) return;
    std::vector<float4> P(n_), Vv(n_), L(n_), Q(n_);
    check(cudaStreamSynchronize(stream_), "sync");
    check(cudaMemcpy(P.data(), d_pos_, sizeof(float4) * n_, cudaMemcpyDeviceToHost), "download(pos)");
    check(cudaMemcpy(Vv.data(), d_vel_, sizeof(float4) * n_, cudaMemcpyDeviceToHost), "download(vel)");
    check(cudaMemcpy(L.data(), d_lvel_, sizeof(float4) * n_, cudaMemcpyDeviceToHost), "download(lvel)");
    check(cudaMemcpy(Q.data(), d_q_, sizeof(float4) * n_, cudaMemcpyDeviceToHost), "download(q)");
    for (int u = 0; u < n_; u++) {
        const int d = u2d_[u];
        pos_[u] = V4{P[d].x, P[d].y, P[d].z, 0.f};
        vel_[u] = V4{Vv[d].x, Vv[d].y, Vv[d].z, 0.f};
        lvel_[u] = V4{L[d].x, L[d].y, L[d].z, 0.f};
        q_[u] = V4{Q[d].x, Q[d].y, Q[d].z, Q[d].w};
    }
    if (host_const_stale_) {  // constants changed by set_parameters live in the .w lanes and qrest
        std::vector<float4> QR(n_);
        check(cudaMemcpy(QR.data(), d_qrest_, sizeof(float4) * n_, cudaMemcpyDeviceToHost), "download(qrest)");
        for (int u = 0; u < n_; u++) {
            const int d = u2d_[u];
            im_[u] = P[d].w;
            ks_[u] = L[d].w;
            qrest_[u] = V4{QR[d].x, QR[d].y, QR[d].z, QR[d].w};
        }
        host_const_stale_ = false;
    }
    host_dyn_valid_ = true;
}

// ------------------------------------------------------------------ host edits
void Batch::set_vertex_inv_mass(int u, float im) {
    ensure_host();
    if (im_[u] != 0.f) im_[u] = im;
    device_valid_ = false;
}
void Batch::set_vertex_ea(int u, float ea) {
    ensure_host();
    ks_[u] = ea * lr_[u];
    device_valid_ = false;
}
void Batch::set_vertex_ei(int u, float ei) {
    ensure_host();
    const float k = 4.f * ei / lr_[u];
    qrest_[u] = scale4(normalize4(qrest_[u]), k);
    device_valid_ = false;
}
void Batch::set_root_host(int rope, const float* p, const float* v, const float* q) {
    ensure_host();
    const int u = ustart_[rope];
    pos_[u] = V4{p[0], p[1], p[2], 0.f};
    vel_[u] = V4{v[0], v[1], v[2], 0.f};
    if (q) q_[u] = V4{q[0], q[1], q[2], q[3]};
    device_valid_ = false;
}
void Batch::set_velocities_host(const float* v) {
    ensure_host();
    for (int u = 0; u < n_; u++) vel_[u] = V4{v[3 * u], v[3 * u + 1], v[3 * u + 2], 0.f};
    device_valid_ = false;
}
void Batch::unpin_root(int rope) {
    ensure_host();
    const int u = ustart_[rope];
    im_[u] = 2.f * im_[u + 1];
    vel_[u] = V4{0.f, 0.f, 0.f, 0.f};
    device_valid_ = false;
}
void Batch::reset_all() {
    ensure_host();
    for (int u = 0; u < n_; u++) {
        pos_[u] = init_pos_[u];
        q_[u] = init_q_[u];
        vel_[u] = V4{0.f, 0.f, 0.f, 0.f};
        lvel_[u] = V4{0.f, 0.f, 0.f, 0.f};
    }
    time_ = 0.f;
    h_ = max_h;
    last_error_ = last_warning_ = 0;
    device_valid_ = false;
    ensure_device();
    gather();
}
void Batch::reset_ropes(const int* ids, int count) {
    if (count <= 0) return;
    ensure_device();
    std::vector<int2> rg(count);
    int maxv = 0;
    for (int c = 0; c < count; c++) {
        const int u = ustart_[ids[c]];
        rg[c] = make_int2(u2d_[u], rope_verts(ids[c]));
        maxv = std::max(maxv, rg[c].y);
    }
    check(cudaMemcpyAsync(d_ranges_, rg.data(), sizeof(int2) * count, cudaMemcpyHostToDevice, stream_), "upload(reset ids)");
    check(launch_reset(d_pos_, d_vel_, d_lvel_, d_q_, d_init_pos_, d_init_q_, d_ranges_, count, maxv, stream_), "reset");
    host_dyn_valid_ = false;
    gather();
    check(cudaStreamSynchronize(stream_), "reset");
}
void Batch::gather() {
    ensure_device();
    FrameArgs a{};
    a.topo = d_topo_; a.pos = d_pos_; a.vel = d_vel_; a.q = d_q_;
    a.out_pos = d_out_pos_; a.out_vel = d_out_vel_; a.out_q = d_out_q_;
    check(launch_gather(a, n_, stream_), "gather");
}
void Batch::download(float* p, float* v, float* q) {
    ensure_host();
    for (int u = 0; u < n_; u++) {
        if (p) { p[3 * u] = pos_[u].x; p[3 * u + 1] = pos_[u].y; p[3 * u + 2] = pos_[u].z; }
        if (v) { v[3 * u] = vel_[u].x; v[3 * u + 1] = vel_[u].y; v[3 * u + 2] = vel_[u].z; }
        if (q) { q[4 * u] = q_[u].x; q[4 * u + 1] = q_[u].y; q[4 * u + 2] = q_[u].z; q[4 * u + 3] = q_[u].w; }
    }
}

// ------------------------------------------------------------------ stepping
// Root rows [R, 17] = (p0, v0, p1, q0, q1) staged into library memory before the launch
// (batch.cu:327-346): callers may free their tensors as soon as the call returns.
void Batch::stage_rows(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1, bool host) {
    if (host) {
        // the previous frame's upload from this pinned buffer must be done before reuse
        check(cudaStreamSynchronize(stream_), "sync(program staging)");
        for (int r = 0; r < R_; r++) {
            float* row = h_prog_ + (size_t)r * 17;
            for (int k = 0; k < 3; k++) {
                row[k] = p0[3 * r + k];
                row[3 + k] = v0[3 * r + k];
                row[6 + k] = p1 ? p1[3 * r + k] : 0.f;
            }
            for (int k = 0; k < 4; k++) {
                row[9 + k] = q0 ? q0[4 * r + k] : 0.f;
                row[13 + k] = q1 ? q1[4 * r + k] : 0.f;
            }
        }
        check(cudaMemcpyAsync(d_prog_, h_prog_, sizeof(float) * 17 * R_, cudaMemcpyHostToDevice, stream_), "upload(program)");
        return;
    }
    const size_t rowb = 17 * sizeof(float);
    check(cudaMemcpy2DAsync(d_prog_, rowb, p0, 3 * sizeof(float), 3 * sizeof(float), R_, cudaMemcpyDeviceToDevice, stream_), "stage p0");
    check(cudaMemcpy2DAsync(d_prog_ + 3, rowb, v0, 3 * sizeof(float), 3 * sizeof(float), R_, cudaMemcpyDeviceToDevice, stream_), "stage v0");
    if (p1) check(cudaMemcpy2DAsync(d_prog_ + 6, rowb, p1, 3 * sizeof(float), 3 * sizeof(float), R_, cudaMemcpyDeviceToDevice, stream_), "stage p1");
    if (q0) check(cudaMemcpy2DAsync(d_prog_ + 9, rowb, q0, 4 * sizeof(float), 4 * sizeof(float), R_, cudaMemcpyDeviceToDevice, stream_), "stage q0");
    if (q1) check(cudaMemcpy2DAsync(d_prog_ + 13, rowb, q1, 4 * sizeof(float), 4 * sizeof(float), R_, cudaMemcpyDeviceToDevice, stream_), "stage q1");
}

// The parameters of one frame launch from the current state (h_ / last_h_ already advanced).
FrameArgs Batch::frame_args(int root_mode, bool has_q0, bool has_q1, float dt, int steps) const {
    FrameArgs a{};
    a.bins = d_bins_; a.ropes = d_ropes_; a.topo = d_topo_;
    a.num_bins = (int)bins_.size();
    a.queue = nullptr; a.order = nullptr; a.bin_cost = nullptr;  // static grid unless run_frame queues
    a.pos = d_pos_; a.vel = d_vel_; a.lvel = d_lvel_; a.q = d_q_; a.qrest = d_qrest_;
    a.out_pos = d_out_pos_; a.out_vel = d_out_vel_; a.out_q = d_out_q_;
    a.out_force = d_force_; a.wrench = d_wrench_; a.status = d_status_;
    a.prog = d_prog_; a.root_mode = root_mode; a.has_q0 = has_q0; a.has_q1 = has_q1;
    a.h = h_; a.last_h = last_h_; a.dt = dt; a.substeps = steps; a.iters = num_itr;
    a.gx = gravity[0]; a.gy = gravity[1]; a.gz = gravity[2];
    a.damping = damping; a.drag = drag; a.drag_quad = drag_quad; a.drag_quad_t = drag_quad_t; a.accel = accel;
    a.num_planes = num_planes_;
    for (int p = 0; p < num_planes_; p++) a.planes[p] = make_float4(planes_[p][0], planes_[p][1], planes_[p][2], planes_[p][3]);
    a.c_radius = c_radius_; a.c_kappa = c_kappa_; a.c_mu_s = c_mu_s_; a.c_mu_k = c_mu_k_; a.c_vslip = c_vslip_;
    a.num_sdf = (int)grids_.size();
    a.sdf_moving = sdf_moving_ ? 1 : 0;
    a.forces_on = forces_on_ ? 1 : 0;
    a.pose_cache = pose_cache_entries();
    a.poses = d_poses_; a.motion = d_motion_;
    for (int m = 0; m < (int)grids_.size(); m++) a.grids[m] = grids_[m];
    a.n = n_;
    a.num_ropes = R_;
    a.rope_contact = rope_contact_ ? 1 : 0;
    a.rc_radius = rc_radius_; a.rc_barrier = rc_barrier_; a.rc_kcol = rc_kcol_; a.rc_mu = rc_mu_; a.rc_kfric = rc_kfric_;
    a.det_radius = rc_radius_ + 0.5f * rc_barrier_;          // uploadMeta, YarnBall.cu:262-263
    a.sdet_radius = a.det_radius * rc_scaler_;
    a.grp = d_grp_; a.cols = d_cols_; a.ncols = d_ncols_; a.maxstep = d_maxstep_; a.pad = d_pad_;
    a.sdf_skip = culling_ ? 1 : 0;
    a.surf_cull = culling_ ? 1 : 0;
    // stage the lattices' block bounds in each CTA's shared memory when they take <= 48 KB and
    // the CTA's shared memory (frame state 144 B per thread, pose cache, bounds) stays <= 200 KB
    const size_t btot = grids_.empty() ? 0 : (size_t)(grids_.back().boff + grids_.back().bcount);
    const size_t smem = (size_t)144 * block_ + (size_t)2 * a.pose_cache * (sizeof(Pose) + 2 * sizeof(float4)) +
                        btot * sizeof(float);
    a.sdf_btab = (btot * sizeof(float) <= 48 * 1024 && smem <= 200 * 1024) ? (int)btot : 0;
    return a;
}

void Batch::run_frame(int root_mode, bool has_q0, bool has_q1, float dt, int steps, float h) {
    // uploadMeta bookkeeping, batch.cu:57-62 / step.cpp:41-42
    last_h_ = h_;
    h_ = h;
    FrameArgs a = frame_args(root_mode, has_q0, has_q1, dt, steps);
    a.tape = pending_tape_;
    a.itape = pending_itape_;
    const bool plain = engine_ == 1 || (rope_contact_ && oversize_);
    const bool queued = queue_ && !plain;
    if (queued) {
        // the previous frame's bin times, if they have arrived, set this frame's order
        if (costs_inflight_) {
            if (cudaEventQuery(ev_cost_) == cudaSuccess) reorder_bins();
            else cudaGetLastError();  // "not ready" is no error: keep the previous order
            costs_inflight_ = false;
        }
        check(cudaMemsetAsync(d_queue_, 0, sizeof(int), stream_), "zero(work queue)");
        a.queue = d_queue_; a.order = d_order_; a.bin_cost = d_bin_cost_;
    }
    const bool timed = timing_ || tuning();
    // a timed frame measures the kernel, not its first-use loading (each trial of the autotuner
    // is the first launch of its bin size)
    if (timed && !plain) check(prepare_frame(a, block_), "frame kernel set-up");
    if (timed) check(cudaEventRecord(ev0_, stream_), "event");
    if (plain) run_frame_plain(a);
    else check(launch_frame(a, block_, (int)bins_.size(), stream_), "frame kernel");
    if (timed) check(cudaEventRecord(ev1_, stream_), "event");
    if (queued && sync_every_frame) {
        check(cudaMemcpyAsync(h_bin_cost_, d_bin_cost_, sizeof(float) * bins_.size(), cudaMemcpyDeviceToHost, stream_),
              "download(bin times)");
        check(cudaEventRecord(ev_cost_, stream_), "event");
        costs_inflight_ = true;
    }
    host_dyn_valid_ = false;
}

// Longest-processing-time-first order of the bins from the last frame's measured times, so the
// work queue hands the slowest bins out first and no slow bin starts last. A counting pass over
// 64 equal-width cost buckets (slowest bucket first, packing order within a bucket) keeps the
// host's turn between frames O(bins): exact LPT is not needed, only no slow bin at the end.
void Batch::reorder_bins() {
    constexpr int kBuckets = 64;
    const int nb = (int)bins_.size();
    float lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < nb; i++) {
        lo = std::min(lo, h_bin_cost_[i]);
        hi = std::max(hi, h_bin_cost_[i]);
    }
    if (!(hi > lo)) return;  // uniform (or unmeasured) bins: keep the order
    const float scale = (kBuckets - 1) / (hi - lo);
    int count[kBuckets + 1] = {};
    order_scratch_.resize(nb);
    for (int i = 0; i < nb; i++) {
        const int k = kBuckets - 1 - std::min(kBuckets - 1, std::max(0, (int)((h_bin_cost_[i] - lo) * scale)));
        order_scratch_[i] = k;
        count[k + 1]++;
    }
    for (int k = 0; k < kBuckets; k++) count[k + 1] += count[k];
    for (int i = 0; i < nb; i++) h_order_[count[order_scratch_[i]]++] = i;
    check(cudaMemcpyAsync(d_order_, h_order_, sizeof(int) * nb, cudaMemcpyHostToDevice, stream_), "upload(bin order)");
}

// The grid broad phase serves contact groups larger than one CTA (the brute force's O(V²) pairs
// per substep dominate there); groups that fit a CTA keep the brute force, as the reference.
const RopeGrid* Batch::rope_grid() {
    if (!oversize_) return nullptr;
    if (!grid_mem_) {
        RopeGrid g{};
        g.T = rope_grid_buckets(n_);
        g.scan_bytes = rope_grid_scan_bytes(g.T);
        const size_t N = (size_t)n_, T = (size_t)g.T;
        // seven sub-buffers, each rounded up to 256 bytes
        const size_t bytes = sizeof(float4) * N + sizeof(int) * (2 * N + 2 * (T + 1)) + sizeof(unsigned) + g.scan_bytes + 8 * 256;
        check(cudaMalloc(&grid_mem_, bytes), "cudaMalloc(rope grid)");
        char* p = static_cast<char*>(grid_mem_);
        auto take = [&](size_t sz) { char* r = p; p += (sz + 255) & ~size_t(255); return r; };
        g.ms = reinterpret_cast<float4*>(take(sizeof(float4) * N));
        g.bucket = reinterpret_cast<int*>(take(sizeof(int) * N));
        g.sorted = reinterpret_cast<int*>(take(sizeof(int) * N));
        g.count = reinterpret_cast<int*>(take(sizeof(int) * (T + 1)));
        g.start = reinterpret_cast<int*>(take(sizeof(int) * (T + 1)));
        g.smax = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
        g.scan_tmp = take(g.scan_bytes);
        grid_ = g;
    }
    return &grid_;
}

// ------------------------------------------------------------------ plain engine
int Batch::bounds_violation() {
    if (!d_status_) return 0;
    int v = 0;
    check(cudaStreamSynchronize(stream_), "sync");
    check(cudaMemcpy(&v, d_status_ + 3, sizeof(int), cudaMemcpyDeviceToHost), "download(status)");
    return v;
}

void Batch::set_engine(int e) {
    if (e != 0 && e != 1) throw std::invalid_argument("engine must be 0 (persistent) or 1 (plain)");
    engine_ = e;
    if (e == 1) autotune_ = false;
}

void Batch::plain_alloc() {
    if (pl_.dx) return;
    const size_t n4 = sizeof(float4) * n_;
    check(cudaMalloc(&pl_.dx, n4), "cudaMalloc(plain dx)");
    check(cudaMalloc(&pl_.dxn, n4), "cudaMalloc(plain dxn)");
    check(cudaMalloc(&pl_.y, n4), "cudaMalloc(plain y)");
    check(cudaMalloc(&pl_.qprev, n4), "cudaMalloc(plain qprev)");
    check(cudaMalloc(&pl_.lpos, n4), "cudaMalloc(plain lpos)");
    check(cudaMalloc(&pl_.facc, n4), "cudaMalloc(plain facc)");
    check(cudaMemset(pl_.facc, 0, n4), "memset(plain facc)");
    check(cudaMalloc(&pl_.cand, sizeof(uint64_t) * n_), "cudaMalloc(plain cand)");
    check(cudaMalloc(&pl_.spose, sizeof(Pose) * (size_t)R_ * kMaxSdf), "cudaMalloc(plain poses)");
    check(cudaMalloc(&d_pl_args_, sizeof(FrameArgs)), "cudaMalloc(plain args)");
    check(cudaMallocHost(&h_pl_args_, sizeof(FrameArgs)), "cudaMallocHost(plain args)");
}

// One frame of the plain path: parameters uploaded once (uploadMeta, YarnBall.cu:261-272),
// then per substep the root / pose / init launches and one replay of the captured iterations.
void Batch::run_frame_plain(const FrameArgs& a) {
    plain_alloc();
    check(cudaStreamSynchronize(stream_), "plain args reuse");  // the previous frame read h_pl_args_
    *h_pl_args_ = a;
    // as the in-repo baseline the plain path samples every candidate lattice, as the reference does;
    // as the product path of contact groups larger than a CTA it keeps the exact block skip
    h_pl_args_->sdf_skip = engine_ == 1 ? 0 : 1;
    check(cudaMemcpyAsync(d_pl_args_, h_pl_args_, sizeof(FrameArgs), cudaMemcpyHostToDevice, stream_), "upload(args)");
    const int surf = a.num_sdf > 0 ? 2 : (a.num_planes > 0 ? 1 : 0);
    const std::string key = std::to_string(a.iters) + ":" + std::to_string(surf) + ":" + std::to_string(a.rope_contact);
    if (!pl_graph_ || key != pl_graph_key_) {
        if (pl_graph_) { cudaGraphExecDestroy(pl_graph_); pl_graph_ = nullptr; }
        cudaGraph_t graph;
        check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
        const cudaError_t rec = plain_record_inner(d_pl_args_, pl_, n_, a.iters, surf, a.rope_contact != 0, stream_);
        check(cudaStreamEndCapture(stream_, &graph), "end capture");
        check(rec, "record plain iterations");
        check(cudaGraphInstantiate(&pl_graph_, graph, 0), "instantiate plain graph");
        cudaGraphDestroy(graph);
        pl_graph_key_ = key;
    }
    for (int s = 0; s < a.substeps; s++) {
        check(plain_launch_pre(d_pl_args_, pl_, n_, R_, R_, a.num_sdf, a.sdf_moving != 0, a.root_mode, a.rope_contact != 0, s,
                               a.rope_contact ? rope_grid() : nullptr, stream_),
              "plain substep prologue");
        check(cudaGraphLaunch(pl_graph_, stream_), "plain graph launch");
    }
    check(plain_launch_finish(d_pl_args_, pl_, n_, stream_), "plain frame end");
}

// ------------------------------------------------------------------ autotuner
namespace {
std::mutex g_tune_mtx;
std::map<std::string, int> g_tune_cache;  // workload signature -> bin size
}  // namespace

std::string Batch::tune_key() const {
    int dev = 0;
    cudaGetDevice(&dev);
    int maxV = 0;
    for (int r = 0; r < R_; r++) maxV = std::max(maxV, rope_verts(r));
    const int surf = grids_.empty() ? (num_planes_ > 0 ? 1 : 0) : 2;
    return std::to_string(dev) + ":" + std::to_string(n_) + ":" + std::to_string(R_) + ":" + std::to_string(maxV) + ":" +
           std::to_string(surf) + ":" + std::to_string(grids_.size()) + ":" + std::to_string(num_itr);
}

void Batch::tune_before_frame() {
    if (!tuning()) return;
    if (tune_cands_.empty()) {
        {
            std::lock_guard<std::mutex> g(g_tune_mtx);
            auto it = g_tune_cache.find(tune_key());
            if (it != g_tune_cache.end()) {
                tuned_ = true;
                if (it->second != block_) { tune_block_ = it->second; ensure_host(); layout_valid_ = false; device_valid_ = false; ensure_device(); }
                return;
            }
        }
        int maxV = 0;
        for (int r = 0; r < R_; r++) maxV = std::max(maxV, rope_verts(r));
        const int lo = std::max(64, next_pow2(maxV));
        const int hi = std::max(256, lo);
        for (int b = lo; b <= hi && b <= 1024; b *= 2) tune_cands_.push_back(b);
        if (tune_cands_.size() < 2) { tuned_ = true; return; }
        // the first candidate again at the end: its first trial is the batch's first frame (first
        // touch of its state), and each candidate keeps its faster trial
        tune_cands_.push_back(tune_cands_.front());
    }
    const int k = (int)tune_log_.size();
    if (k < (int)tune_cands_.size() && tune_cands_[k] != block_) {
        tune_block_ = tune_cands_[k];
        ensure_host();
        layout_valid_ = false;
        device_valid_ = false;
        ensure_device();
    }
}

void Batch::tune_after_frame() {
    if (!tuning() || tune_cands_.empty()) return;
    check(cudaEventSynchronize(ev1_), "tune sync");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed");
    tune_log_.push_back({block_, (double)ms});
    if (tune_log_.size() < tune_cands_.size()) return;
    std::map<int, double> trial;  // bin size -> its faster trial
    for (const auto& e : tune_log_) {
        auto it = trial.find(e.first);
        if (it == trial.end() || e.second < it->second) trial[e.first] = e.second;
    }
    auto best = std::min_element(trial.begin(), trial.end(),
                                 [](const std::pair<const int, double>& x, const std::pair<const int, double>& y) {
                                     return x.second < y.second;
                                 });
    // Ties within 3% (the trial frames are different frames of the run) go to the smallest bins:
    // they spread a frame over more CTAs, and the adjoint, which runs on the forward's bins, gains
    // from that (1024 64-vertex ropes: 37.0 against 38.3 ms per 30 reverses in 64- and 128-thread
    // bins, at 20.9 and 21.1 ms per 30 forward frames).
    const double limit = best->second * 1.03;
    for (auto it = trial.begin(); it != trial.end(); ++it)
        if (it->second <= limit && it->first < best->first) best = it;
    tuned_ = true;
    {
        std::lock_guard<std::mutex> g(g_tune_mtx);
        g_tune_cache[tune_key()] = best->first;
    }
    if (best->first != block_) {
        tune_block_ = best->first;
        ensure_host();
        layout_valid_ = false;
        device_valid_ = false;
        ensure_device();
        gather();
    }
}

void Batch::sdf_begin() {
    if (pending_set_) {
        check(launch_stage_motion(d_cur_, d_tgt_, d_tele_, d_motion_, R_ * kMaxSdf, stream_), "stage motion");
        sdf_moving_ = true;
        moving_ = true;
    } else {
        sdf_moving_ = false;
    }
    if (forces_on_) {
        check(cudaMemsetAsync(d_force_, 0, sizeof(float) * 3 * n_, stream_), "zero(contact forces)");
        check(cudaMemsetAsync(d_wrench_, 0, sizeof(float) * 6 * (size_t)R_ * kMaxSdf, stream_), "zero(mesh wrenches)");
    }
}

void Batch::sdf_end(int substeps) {
    last_substeps_ = substeps > 0 ? substeps : 1;
    if (moving_) {
        check(launch_commit(d_cur_, d_tgt_, d_tele_, d_poses_, d_boxes_, (int)grids_.size(), -1, R_, stream_), "commit poses");
        moving_ = false;
        pending_set_ = false;
    }
    if (forces_on_)
        check(launch_scale(d_wrench_, 6 * R_ * kMaxSdf, 1.f / (float)last_substeps_, stream_), "average wrenches");
}

void Batch::step_program(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1, float dt,
                         int substeps, bool host_inputs) {
    tune_before_frame();
    ensure_device();
    stage_rows(p0, v0, p1, q0, q1, host_inputs);
    sdf_begin();
    run_frame(ROOT_PROGRAM, q0 != nullptr, q1 != nullptr, dt, substeps, dt / (float)substeps);
    time_ += dt;
    sdf_end(substeps);
    tune_after_frame();
    if (sync_every_frame) {
        check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
        check(cudaStreamSynchronize(stream_), "frame");
        if (h_status_[0] || h_status_[1] || h_status_[2]) {
            if (h_status_[2]) nonfinite_ = 1;
            if (h_status_[1]) last_warning_ = h_status_[1];
            const int err = h_status_[0];
            check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
            if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        }
    }
    if (timing_) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed");
        last_frame_ms_ = ms;
    }
}

// A program-driven frame that calls no device allocator: the rope-rope candidate lists go to the
// library's static device array (static_scratch_cols) instead of the handle's own buffer, and
// every step that could allocate (autotuning repacks, a pending upload, the plain engine) is
// refused up front instead of performed.
void Batch::step_program_static_scratch(const float* p0, const float* v0, const float* p1, const float* q0,
                                        const float* q1, float dt, int substeps) {
    int* cols = nullptr;
    int cap = 0;
    check(static_scratch_cols(&cols, &cap), "static scratch address");
    if (n_ > cap)
        throw std::invalid_argument("the allocation-free step's static scratch holds at most " + std::to_string(cap) +
                                    " vertices; this batch has " + std::to_string(n_));
    if (engine_ != 0) throw std::invalid_argument("the allocation-free step runs the persistent engine only");
    if (!layout_valid_ || !device_valid_)
        throw std::invalid_argument("host-side edits are pending upload: run one regular step (or gather) first");
    if (rope_contact_ && oversize_)
        throw std::invalid_argument("a rope-rope contact group larger than one CTA needs the plain engine, which allocates");
    stage_rows(p0, v0, p1, q0, q1, false);
    sdf_begin();
    last_h_ = h_;
    h_ = dt / (float)substeps;
    FrameArgs a = frame_args(ROOT_PROGRAM, q0 != nullptr, q1 != nullptr, dt, substeps);
    a.cols = cols;
    if (timing_) check(cudaEventRecord(ev0_, stream_), "event");
    check(launch_frame(a, block_, (int)bins_.size(), stream_), "frame kernel");
    if (timing_) check(cudaEventRecord(ev1_, stream_), "event");
    host_dyn_valid_ = false;
    time_ += dt;
    sdf_end(substeps);
    check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
    check(cudaStreamSynchronize(stream_), "frame");
    if (h_status_[0] || h_status_[1] || h_status_[2]) {
        if (h_status_[2]) nonfinite_ = 1;
        if (h_status_[1]) last_warning_ = h_status_[1];
        const int err = h_status_[0];
        check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
        if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
    }
    if (timing_) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed");
        last_frame_ms_ = ms;
    }
}

void Batch::step_legacy(const float* p, const float* v, const float* q, float dt, int substeps, bool host_inputs) {
    tune_before_frame();
    ensure_device();
    stage_rows(p, v, nullptr, q, nullptr, host_inputs);
    sdf_begin();
    // exactly `substeps` substeps through the biased max_h of batch.cu:306-308 (float ceil)
    const float mh = (dt / (float)substeps) * 1.000001f;
    int steps = (int)std::ceil(dt / mh);
    if (steps < 1) steps = 1;
    run_frame(ROOT_SET, q != nullptr, false, dt, steps, dt / (float)steps);
    time_ += dt;
    sdf_end(substeps);
    tune_after_frame();
    if (sync_every_frame) {
        check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
        check(cudaStreamSynchronize(stream_), "frame");
        if (h_status_[0] || h_status_[2]) {
            if (h_status_[2]) nonfinite_ = 1;
            const int err = h_status_[0];
            check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
            if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        }
    }
    if (timing_) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev0_, ev1_), "elapsed");
        last_frame_ms_ = ms;
    }
}

void Batch::step_free(float dt, int substeps) {
    tune_before_frame();
    ensure_device();
    sdf_begin();
    run_frame(ROOT_NONE, false, false, dt, substeps, dt / (float)substeps);
    time_ += dt;
    sdf_end(substeps);
    tune_after_frame();
    if (sync_every_frame) {
        check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
        check(cudaStreamSynchronize(stream_), "frame");
        if (h_status_[0] || h_status_[2]) {
            if (h_status_[2]) nonfinite_ = 1;
            const int err = h_status_[0];
            check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
            if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        }
    }
}

// Sim::advance (step.cpp:37-57) with bindings.cpp:274-295's explicit-substep bias.
void Batch::advance(float dt, int substeps) {
    if (!(dt > 0.f)) return;
    tune_before_frame();
    ensure_device();
    sdf_begin();
    const float mh = substeps > 0 ? (dt / (float)substeps) * 1.000001f : max_h;
    int steps = (int)std::ceil(dt / mh);
    if (steps < 1) steps = 1;
    run_frame(ROOT_NONE, false, false, dt, steps, dt / (float)steps);
    time_ += dt;
    sdf_end(substeps > 0 ? substeps : steps);
    tune_after_frame();
    if (sync_every_frame) {
        check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
        check(cudaStreamSynchronize(stream_), "frame");
        if (h_status_[0] || h_status_[2]) {
            if (h_status_[2]) nonfinite_ = 1;
            const int err = h_status_[0];
            check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
            if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        }
    }
}

void Batch::set_rope_contact(bool on, float radius, float barrier, float k_collision, float mu, float k_friction,
                             float detection_scaler, int group_ropes) {
    if (on) {
        // uploadMeta enforces this every step (YarnBall.cu:268): check it here so a bad call
        // leaves the old state (batch.cu:372-375)
        if (2.f * min_seg_ < 2.f * radius + barrier)
            throw std::invalid_argument("rope contact needs 2 * radius + barrier <= 2 * shortest segment");
        if (!(detection_scaler > 1.f)) throw std::invalid_argument("Detection scaler must be greater than 1.");
    }
    ensure_host();
    const bool relayout = on != rope_contact_ || (on && group_ropes != group_ropes_);
    if (on) {
        rc_radius_ = radius; rc_barrier_ = barrier; rc_kcol_ = k_collision; rc_mu_ = mu; rc_kfric_ = k_friction;
        rc_scaler_ = detection_scaler;
        group_ropes_ = group_ropes > 0 ? group_ropes : 1;
        if (!d_cols_) {
            check(cudaMalloc(&d_cols_, sizeof(int) * (size_t)kMaxCols * n_), "cudaMalloc(rope candidates)");
            check(cudaMalloc(&d_ncols_, sizeof(int) * n_), "cudaMalloc(rope candidate counts)");
            check(cudaMalloc(&d_maxstep_, sizeof(float) * n_), "cudaMalloc(step limits)");
            check(cudaMalloc(&d_pad_, sizeof(float) * n_), "cudaMalloc(paddings)");
            check(cudaMemset(d_ncols_, 0, sizeof(int) * n_), "memset(rope candidate counts)");
        }
    }
    rope_contact_ = on;
    if (relayout) {
        layout_valid_ = false;
        device_valid_ = false;
        tuned_ = false;
        tune_cands_.clear();
        tune_log_.clear();
        tune_block_ = 0;
        ensure_device();
        gather();
    }
}

void Batch::set_block(int block) {
    if (block == block_override) return;
    ensure_host();
    block_override = block;
    layout_valid_ = false;
    device_valid_ = false;
    ensure_device();
    gather();
}

// ------------------------------------------------------------------ contact
void Batch::set_contact(float radius, float mu_s, float mu_k, float v_slip, float kappa) {
    c_radius_ = radius; c_mu_s_ = mu_s; c_mu_k_ = mu_k; c_vslip_ = v_slip; c_kappa_ = kappa;
    refresh_contact_boxes();
}
// The union of the lattice blocks whose lower bound does not clear the contact radius: outside
// it no probe can reach gap < 0 (the persistent kernel's exact per-iteration rejection).
void Batch::refresh_contact_boxes() {
    for (size_t m = 0; m < grids_.size(); m++) {
        GridDesc& g = grids_[m];
        const std::vector<float>& b = bmin_host_[m];
        const int bx = (g.nx - 2) / kSdfBlock + 1;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        const int n[3] = {g.nx, g.ny, g.nz}, bn[3] = {bx, g.by, g.bz};
        const float o[3] = {g.ox, g.oy, g.oz};
        bool any = false;
        for (int i = 0; i < bn[0]; i++)
            for (int j = 0; j < bn[1]; j++)
                for (int k = 0; k < bn[2]; k++) {
                    if (b[((size_t)i * g.by + j) * g.bz + k] - c_radius_ > 1e-5f) continue;
                    any = true;
                    const int ijk[3] = {i, j, k};
                    for (int a = 0; a < 3; a++) {
                        lo[a] = std::min(lo[a], o[a] + float(ijk[a] * kSdfBlock) * g.h);
                        hi[a] = std::max(hi[a], o[a] + float(std::min(ijk[a] * kSdfBlock + kSdfBlock, n[a] - 1)) * g.h);
                    }
                }
        g.never = any ? 0 : 1;
        for (int a = 0; a < 3; a++) {
            g.tlo[a] = any ? lo[a] - 1e-4f : 0.f;
            g.thi[a] = any ? hi[a] + 1e-4f : 0.f;
        }
    }
}
void Batch::set_planes(int count, const float* rows) {
    for (int p = 0; p < count; p++)
        for (int k = 0; k < 4; k++) planes_[p][k] = rows[4 * p + k];
    num_planes_ = count;
}

// 1 / L for the trilinear interpolant of a lattice: within a cell d(phi)/dx is a bilinear blend of
// the cell's four x-edge differences over the spacing, so |d(phi)/dx| <= Dx (the largest x-edge
// difference of the lattice over the spacing), likewise y and z, and the interpolant (continuous
// across cells) is Lipschitz with L = |(Dx, Dy, Dz)|. Accumulated in double, L is rounded up and
// 1 / L down; a constant field gives a large finite value.
static float lattice_lipschitz_inv(const float* v, int nx, int ny, int nz, float spacing) {
    double D[3] = {0.0, 0.0, 0.0};
    auto at = [&](int i, int j, int k) { return (double)v[((size_t)i * ny + j) * nz + k]; };
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const double c = at(i, j, k);
                if (i + 1 < nx) D[0] = std::max(D[0], std::fabs(at(i + 1, j, k) - c));
                if (j + 1 < ny) D[1] = std::max(D[1], std::fabs(at(i, j + 1, k) - c));
                if (k + 1 < nz) D[2] = std::max(D[2], std::fabs(at(i, j, k + 1) - c));
            }
    const double L = std::sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]) / (double)spacing * (1.0 + 1e-6);
    const double inv = 1.0 / std::max(L, 1e-6);
    return std::nextafter((float)inv, 0.f);
}

int Batch::add_mesh(const float* values, int nx, int ny, int nz, const float* origin, float spacing, float mu_s,
                    float mu_k, const float* pos, const float* quat, int rows) {
    if ((int)grids_.size() >= kMaxSdf) throw std::invalid_argument("at most 64 meshes per sim");
    ensure_device();
    const size_t cnt = (size_t)nx * ny * nz;
    float* d = nullptr;
    check(cudaMalloc(&d, sizeof(float) * cnt), "cudaMalloc(sdf grid)");
    const cudaError_t e = cudaMemcpy(d, values, sizeof(float) * cnt, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(d); check(e, "upload(sdf grid)"); }
    GridDesc g{};
    g.v = d; g.nx = nx; g.ny = ny; g.nz = nz;
    g.ox = origin[0]; g.oy = origin[1]; g.oz = origin[2];
    g.h = spacing; g.invH = 1.f / spacing; g.muS = mu_s; g.muK = mu_k;
    // lower bounds of the field per block of kSdfBlock^3 cells (the persistent kernel's exact
    // early out; the block's face nodes are shared with its neighbours)
    const int bnx = (nx - 2) / kSdfBlock + 1, by = (ny - 2) / kSdfBlock + 1, bz = (nz - 2) / kSdfBlock + 1;
    std::vector<float> bmin((size_t)bnx * by * bz, std::numeric_limits<float>::infinity());
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const float val = values[((size_t)i * ny + j) * nz + k];
                // node i belongs to the blocks of cells i - 1 and i
                for (int ci = std::max(0, i - 1); ci <= std::min(i, nx - 2); ci++)
                    for (int cj = std::max(0, j - 1); cj <= std::min(j, ny - 2); cj++)
                        for (int ck = std::max(0, k - 1); ck <= std::min(k, nz - 2); ck++) {
                            float& m = bmin[((size_t)(ci / kSdfBlock) * by + cj / kSdfBlock) * bz + ck / kSdfBlock];
                            m = std::min(m, val);
                        }
            }
    float* db = nullptr;
    const cudaError_t e2 = cudaMalloc(&db, sizeof(float) * bmin.size());
    if (e2 != cudaSuccess) { cudaFree(d); check(e2, "cudaMalloc(sdf block bounds)"); }
    const cudaError_t e3 = cudaMemcpy(db, bmin.data(), sizeof(float) * bmin.size(), cudaMemcpyHostToDevice);
    if (e3 != cudaSuccess) { cudaFree(d); cudaFree(db); check(e3, "upload(sdf block bounds)"); }
    g.bmin = db; g.by = by; g.bz = bz;
    g.lip_inv = lattice_lipschitz_inv(values, nx, ny, nz, spacing);
    g.status = d_status_;
    g.bcount = (int)bmin.size();
    g.boff = grids_.empty() ? 0 : grids_.back().boff + grids_.back().bcount;
    grids_.push_back(g);
    bmin_host_.push_back(std::move(bmin));
    refresh_contact_boxes();
    const float bx[6] = {origin[0], origin[1], origin[2], origin[0] + float(nx - 1) * spacing,
                         origin[1] + float(ny - 1) * spacing, origin[2] + float(nz - 1) * spacing};
    boxes_.insert(boxes_.end(), bx, bx + 6);
    const int idx = (int)grids_.size() - 1;
    check(cudaMemcpyAsync(d_boxes_, boxes_.data(), sizeof(float) * boxes_.size(), cudaMemcpyHostToDevice, stream_), "upload(boxes)");
    const bool pending = pending_set_;
    set_mesh_targets(idx, pos, quat, rows, nullptr, true, false);
    check(launch_commit(d_cur_, d_tgt_, d_tele_, d_poses_, d_boxes_, (int)grids_.size(), idx, R_, stream_), "commit mesh");
    check(cudaStreamSynchronize(stream_), "add_mesh");
    pending_set_ = pending;
    // the per-CTA pose cache must still fit: repack with fewer ropes per bin if needed
    const int M = (int)grids_.size();
    const int cap = std::max(1, (96 * 1024) / (2 * M * (int)(sizeof(Pose) + 2 * sizeof(float4))));
    if (max_rcount_ > cap) {
        ensure_host();
        layout_valid_ = false;
        device_valid_ = false;
        ensure_device();
    }
    return idx;
}

void Batch::set_mesh_friction(int index, float mu_s, float mu_k) {
    if (index < 0 || index >= (int)grids_.size()) throw std::invalid_argument("mesh index out of range");
    grids_[index].muS = mu_s;
    grids_[index].muK = mu_k;
}

void Batch::set_mesh_targets(int index, const float* pos, const float* quat, int rows, const uint8_t* tele, bool tele_all,
                             bool on_device, bool tele_on_host) {
    const int M = (int)grids_.size();
    if (index >= M || (index < 0 && M == 0)) throw std::invalid_argument("mesh index out of range");
    ensure_device();
    const float* dp = pos;
    const float* dq = quat;
    const uint8_t* dt = tele;
    const int nrows = index < 0 ? R_ * M : rows;
    if (!on_device) {
        float* sq = d_stage_ + 3 * (size_t)R_ * kMaxSdf;
        check(cudaMemcpyAsync(d_stage_, pos, sizeof(float) * 3 * nrows, cudaMemcpyHostToDevice, stream_), "upload(target pos)");
        check(cudaMemcpyAsync(sq, quat, sizeof(float) * 4 * nrows, cudaMemcpyHostToDevice, stream_), "upload(target quat)");
        dp = d_stage_;
        dq = sq;
        if (tele && !tele_all) {
            check(cudaMemcpyAsync(d_stage_tele_, tele, R_, cudaMemcpyHostToDevice, stream_), "upload(teleport flags)");
            dt = d_stage_tele_;
        } else {
            dt = nullptr;
        }
        // pageable sources: wait so the caller's arrays may die after the call
        check(cudaStreamSynchronize(stream_), "stage targets");
    } else if (tele_on_host && tele && !tele_all) {
        // device poses with host teleport flags: stage the flags
        check(cudaMemcpyAsync(d_stage_tele_, tele, R_, cudaMemcpyHostToDevice, stream_), "upload(teleport flags)");
        check(cudaStreamSynchronize(stream_), "stage teleport flags");
        dt = d_stage_tele_;
    }
    check(launch_scatter_targets(d_tgt_, d_tele_, index, dp, dq, rows, M, tele_all ? nullptr : dt, tele_all ? 1 : 0, R_,
                                 stream_),
          "set_mesh_poses");
    pending_set_ = true;
}

void Batch::clear_meshes() {
    check(cudaStreamSynchronize(stream_), "clear_meshes");
    for (auto& g : grids_) {
        cudaFree(const_cast<float*>(g.v));
        cudaFree(const_cast<float*>(g.bmin));
    }
    grids_.clear();
    bmin_host_.clear();
    boxes_.clear();
    pending_set_ = false;
    moving_ = false;
}

void Batch::enable_forces(bool on) {
    if (on && !d_force_) {
        check(cudaMalloc(&d_force_, sizeof(float) * 3 * n_), "cudaMalloc(contact forces)");
        check(cudaMalloc(&d_wrench_, sizeof(float) * 6 * (size_t)R_ * kMaxSdf), "cudaMalloc(mesh wrenches)");
        check(cudaMemset(d_force_, 0, sizeof(float) * 3 * n_), "memset(contact forces)");
        check(cudaMemset(d_wrench_, 0, sizeof(float) * 6 * (size_t)R_ * kMaxSdf), "memset(mesh wrenches)");
    }
    forces_on_ = on;
}

void Batch::contact_forces_host(float* out) {
    if (!forces_on_ || !d_force_) throw std::invalid_argument("enable_contact_forces(True) first");
    check(cudaStreamSynchronize(stream_), "sync");
    check(cudaMemcpy(out, d_force_, sizeof(float) * 3 * n_, cudaMemcpyDeviceToHost), "download(contact forces)");
}

void Batch::wrenches_host(float* out) {
    if (!forces_on_ || !d_wrench_) throw std::invalid_argument("enable_contact_forces(True) first");
    std::vector<float> w(6 * (size_t)R_ * kMaxSdf);
    check(cudaStreamSynchronize(stream_), "sync");
    check(cudaMemcpy(w.data(), d_wrench_, sizeof(float) * w.size(), cudaMemcpyDeviceToHost), "download(mesh wrenches)");
    const int M = (int)grids_.size();
    for (int e = 0; e < R_; e++)
        for (int m = 0; m < M; m++)
            for (int k = 0; k < 6; k++) out[((size_t)e * M + m) * 6 + k] = w[((size_t)e * kMaxSdf + m) * 6 + k];
}

// ------------------------------------------------------------------ differentiable frames
void Batch::grad_alloc(int substeps) {
    const size_t n4 = sizeof(float4) * n_;
    if (!gs_pos_) {
        check(cudaMalloc(&gs_pos_, n4), "cudaMalloc(replay pos)");
        check(cudaMalloc(&gs_vel_, n4), "cudaMalloc(replay vel)");
        check(cudaMalloc(&gs_lvel_, n4), "cudaMalloc(replay lvel)");
        check(cudaMalloc(&gs_q_, n4), "cudaMalloc(replay q)");
        check(cudaMalloc(&gs_buf_, sizeof(float) * 13 * n_), "cudaMalloc(replay views)");
    }
    if (substeps > tape_steps_) {
        if (d_tape_) {
            check(cudaStreamSynchronize(stream_), "tape reuse");
            cudaFree(d_tape_);
            d_tape_ = nullptr;
        }
        check(cudaMalloc(&d_tape_, n4 * 4 * (size_t)substeps), "cudaMalloc(substep tape)");
        tape_steps_ = substeps;
    }
}

void Batch::set_state(const float* pos, const float* vel, const float* lvel, const float* q, bool on_device) {
    ensure_device();
    grad_alloc(0);
    const float *p = pos, *v = vel, *l = lvel, *qq = q;
    if (!on_device) {  // stage host rows through the replay buffer
        check(cudaStreamSynchronize(stream_), "staging reuse");
        float* b = gs_buf_;
        if (pos) check(cudaMemcpy(b, pos, sizeof(float) * 3 * n_, cudaMemcpyHostToDevice), "upload(state pos)"), p = b;
        if (vel) check(cudaMemcpy(b + 3 * n_, vel, sizeof(float) * 3 * n_, cudaMemcpyHostToDevice), "upload(state vel)"), v = b + 3 * n_;
        if (lvel) check(cudaMemcpy(b + 6 * n_, lvel, sizeof(float) * 3 * n_, cudaMemcpyHostToDevice), "upload(state lvel)"), l = b + 6 * n_;
        if (q) check(cudaMemcpy(b + 9 * n_, q, sizeof(float) * 4 * n_, cudaMemcpyHostToDevice), "upload(state q)"), qq = b + 9 * n_;
    }
    check(launch_state_in(d_topo_, p, v, l, qq, d_pos_, d_vel_, d_lvel_, d_pos_, d_vel_, d_lvel_, d_q_, n_, stream_), "set state");
    host_dyn_valid_ = false;
    gather();
    check(cudaStreamSynchronize(stream_), "set state");
}

void Batch::get_state(float* pos, float* vel, float* lvel, float* q, bool on_device) {
    ensure_device();
    if (on_device) {
        check(launch_state_out(d_topo_, d_pos_, d_vel_, d_lvel_, d_q_, pos, vel, lvel, q, n_, stream_), "get state");
        check(cudaStreamSynchronize(stream_), "get state");
        return;
    }
    ensure_host();
    for (int u = 0; u < n_; u++) {
        if (pos) { pos[3 * u] = pos_[u].x; pos[3 * u + 1] = pos_[u].y; pos[3 * u + 2] = pos_[u].z; }
        if (vel) { vel[3 * u] = vel_[u].x; vel[3 * u + 1] = vel_[u].y; vel[3 * u + 2] = vel_[u].z; }
        if (lvel) { lvel[3 * u] = lvel_[u].x; lvel[3 * u + 1] = lvel_[u].y; lvel[3 * u + 2] = lvel_[u].z; }
        if (q) { q[4 * u] = q_[u].x; q[4 * u + 1] = q_[u].y; q[4 * u + 2] = q_[u].z; q[4 * u + 3] = q_[u].w; }
    }
}

void Batch::set_parameters(const float* ea, const float* ei, const float* mass, bool on_device) {
    if (!on_device) {  // host values are validated and applied through the host mirror
        ensure_host();
        for (int u = 0; u < n_; u++) {
            const bool seg = (fl_[u] & F_NEXT) != 0;
            if (ea && seg && !(ea[u] > 0.f && std::isfinite(ea[u]))) throw std::invalid_argument("ea must be finite and > 0");
            if (ei && seg && !(ei[u] > 0.f && std::isfinite(ei[u]))) throw std::invalid_argument("ei must be finite and > 0");
            if (mass && im_[u] != 0.f && !(mass[u] > 0.f && std::isfinite(mass[u])))
                throw std::invalid_argument("mass must be finite and > 0");
        }
        for (int u = 0; u < n_; u++) {
            const bool seg = (fl_[u] & F_NEXT) != 0;
            if (ea && seg) ks_[u] = ea[u] * lr_[u];
            if (ei && seg) qrest_[u] = scale4(normalize4(qrest_[u]), 4.f * ei[u] / lr_[u]);
            if (mass && im_[u] != 0.f) im_[u] = 1.f / mass[u];
        }
        device_valid_ = false;
        ensure_device();
        return;
    }
    ensure_device();
    check(launch_params_in(d_topo_, ea, ei, mass, d_pos_, d_vel_, d_lvel_, d_qrest_, d_qdir_, n_, stream_), "set parameters");
    check(cudaStreamSynchronize(stream_), "set parameters");
    host_const_stale_ = true;
}

void Batch::get_parameters(float* ea, float* ei, float* mass, bool on_device) {
    ensure_device();
    if (on_device) {
        check(launch_params_out(d_topo_, d_pos_, d_vel_, d_lvel_, d_qrest_, ea, ei, mass, n_, stream_), "get parameters");
        check(cudaStreamSynchronize(stream_), "get parameters");
        return;
    }
    ensure_host();
    for (int u = 0; u < n_; u++) {
        const bool seg = (fl_[u] & F_NEXT) != 0;
        if (ea) ea[u] = seg ? ks_[u] / lr_[u] : 0.f;
        if (ei) {
            const V4 r = qrest_[u];
            ei[u] = seg ? std::sqrt(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w) * lr_[u] * 0.25f : 0.f;
        }
        if (mass) mass[u] = im_[u] != 0.f ? 1.f / im_[u] : 0.f;
    }
}

void Batch::step_program_taped(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1,
                               float dt, int substeps, float* tape) {
    if (!tape) throw std::invalid_argument("null tape");
    if (!grids_.empty() && pending_set_) throw std::invalid_argument("the adjoint differentiates static meshes only: no mesh pose targets may be pending in a differentiated frame");
    pending_tape_ = reinterpret_cast<float4*>(tape);
    try {
        step_program(p0, v0, p1, q0, q1, dt, substeps, false);
    } catch (...) {
        pending_tape_ = nullptr;
        throw;
    }
    pending_tape_ = nullptr;
}

float Batch::frame_forward(const FrameIO& io, float dt, int substeps, bool synchronize) {
    if (!(dt > 0.f)) throw std::invalid_argument("dt must be > 0");
    if (substeps < 1) throw std::invalid_argument("substeps must be >= 1");
    if (!io.pos || !io.vel || !io.lvel || !io.q) throw std::invalid_argument("the frame-start state is required");
    if ((io.p0 != nullptr) != (io.v0 != nullptr) || (io.p0 != nullptr) != (io.p1 != nullptr))
        throw std::invalid_argument("a program frame needs p0, v0 and p1 (all NULL: a free frame)");
    if (!io.o_pos || !io.o_vel || !io.o_lvel || !io.o_q) throw std::invalid_argument("the end-state outputs are required");
    if (io.p0 && !roots_pinned()) throw std::invalid_argument("the program frame drives every rope's root");
    if (io.tape) {
        if (!grids_.empty() && pending_set_) throw std::invalid_argument("the adjoint differentiates static meshes only: no mesh pose targets may be pending in a differentiated frame");
    }
    tune_before_frame();
    ensure_device();
    check(launch_state_in(d_topo_, io.pos, io.vel, io.lvel, io.q, d_pos_, d_vel_, d_lvel_, d_pos_, d_vel_, d_lvel_, d_q_, n_,
                          stream_), "frame state");
    if (io.ea || io.ei || io.mass) {
        check(launch_params_in(d_topo_, io.ea, io.ei, io.mass, d_pos_, d_vel_, d_lvel_, d_qrest_, d_qdir_, n_, stream_),
              "frame parameters");
        host_const_stale_ = true;
    }
    if (io.p0) stage_rows(io.p0, io.v0, io.p1, nullptr, nullptr, false);
    sdf_begin();
    const float last = h_;
    pending_tape_ = reinterpret_cast<float4*>(io.tape);
    pending_itape_ = (io.tape && itape_usable()) ? reinterpret_cast<float4*>(io.itape) : nullptr;
    run_frame(io.p0 ? ROOT_PROGRAM : ROOT_NONE, false, false, dt, substeps, dt / (float)substeps);
    pending_tape_ = nullptr;
    pending_itape_ = nullptr;
    time_ += dt;
    sdf_end(substeps);
    tune_after_frame();
    check(launch_state_out(d_topo_, d_pos_, d_vel_, d_lvel_, d_q_, io.o_pos, io.o_vel, io.o_lvel, io.o_q, n_, stream_),
          "frame outputs");
    if (synchronize) {
        check(cudaMemcpyAsync(h_status_, d_status_, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream_), "status");
        check(cudaStreamSynchronize(stream_), "frame");
        if (h_status_[0] || h_status_[1] || h_status_[2]) {
            if (h_status_[2]) nonfinite_ = 1;
            if (h_status_[1]) last_warning_ = h_status_[1];
            const int err = h_status_[0];
            check(cudaMemsetAsync(d_status_, 0, sizeof(int) * 4, stream_), "reset status");
            if (err) { last_error_ = err; throw solver_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        }
    }
    return last;
}

void Batch::backward(const BackwardIO& io, float dt, int substeps, float last_h, bool synchronize) {
    if (!(dt > 0.f)) throw std::invalid_argument("dt must be > 0");
    if (substeps < 1) throw std::invalid_argument("substeps must be >= 1");
    if (!(last_h > 0.f)) throw std::invalid_argument("last_h must be > 0");
    if (!io.pos || !io.vel || !io.lvel || !io.q) throw std::invalid_argument("the frame-start state (pos, vel, lvel, q) is required");
    if (!io.o_pos || !io.o_vel || !io.o_lvel || !io.o_q) throw std::invalid_argument("the state adjoint outputs are required");
    if (io.p0 && (!io.v0 || !io.p1)) throw std::invalid_argument("a program frame needs p0, v0 and p1");
    if (io.q1 && !io.q0) throw std::invalid_argument("root_q_end requires root_q");
    if (!grids_.empty() && (pending_set_ || sdf_moving_)) throw std::invalid_argument("the adjoint differentiates static meshes only: no mesh pose targets may be pending in a differentiated frame");
    ensure_device();
    // contact groups larger than one CTA (and the plain engine) take the per-launch adjoint
    const bool plain = engine_ == 1 || (rope_contact_ && oversize_);
    if (!plain && block_ > 512)
        throw std::invalid_argument("the adjoint runs bins of at most 512 vertices (ropes of at most 512 vertices)");
    if (!plain &&
        adjoint_smem_bytes(block_, num_itr, rope_contact_) + (size_t)pose_cache_entries() * 5 * sizeof(float4) > 227 * 1024)
        throw std::invalid_argument("num_itr too large for the adjoint's shared memory at this bin size");
    grad_alloc(io.tape ? 0 : substeps);
    if (io.ea || io.ei || io.mass) {
        check(launch_params_in(d_topo_, io.ea, io.ei, io.mass, d_pos_, d_vel_, d_lvel_, d_qrest_, d_qdir_, n_, stream_),
              "backward parameters");
        host_const_stale_ = true;
    }
    if (io.p0) stage_rows(io.p0, io.v0, io.p1, io.q0, io.q1, false);
    FrameArgs a = frame_args(io.p0 ? ROOT_PROGRAM : ROOT_NONE, io.q0 != nullptr, io.q1 != nullptr, dt, substeps);
    a.h = dt / (float)substeps;
    a.last_h = last_h;
    const float4* tape = reinterpret_cast<const float4*>(io.tape);
    if (!tape) {  // replay the frame from its start state to record the tape
        check(launch_state_in(d_topo_, io.pos, io.vel, io.lvel, io.q, d_pos_, d_vel_, d_lvel_, gs_pos_, gs_vel_, gs_lvel_,
                              gs_q_, n_, stream_), "replay state");
        FrameArgs r = a;
        r.pos = gs_pos_; r.vel = gs_vel_; r.lvel = gs_lvel_; r.q = gs_q_;
        r.out_pos = gs_buf_; r.out_vel = gs_buf_ + 3 * (size_t)n_; r.out_q = gs_buf_ + 6 * (size_t)n_;
        r.forces_on = 0; r.out_force = nullptr; r.wrench = nullptr;
        r.tape = d_tape_;
        if (plain) run_frame_plain(r);
        else check(launch_frame(r, block_, (int)bins_.size(), stream_), "frame replay");
        tape = d_tape_;
    }
    AdjArgs g{};
    g.tape = tape;
    // the iterates recorded with this frame's tape (never with a replayed tape)
    g.itape = (io.tape && io.itape && itape_usable()) ? reinterpret_cast<const float4*>(io.itape) : nullptr;
    g.g_pos = io.g_pos; g.g_vel = io.g_vel; g.g_lvel = io.g_lvel; g.g_q = io.g_q;
    g.o_pos = io.o_pos; g.o_vel = io.o_vel; g.o_lvel = io.o_lvel; g.o_q = io.o_q;
    g.o_ea = io.o_ea; g.o_ei = io.o_ei; g.o_mass = io.o_mass;
    g.o_p0 = io.o_p0; g.o_v0 = io.o_v0; g.o_p1 = io.o_p1;
    // o_p0 / o_v0 / o_p1: every rope's first vertex (F_ROOT) writes its rope's row in the adjoint
    if (plain) {
        const size_t words = adjoint_plain_words(n_, num_itr);
        if (words > padj_words_) {
            if (d_padj_) check(cudaStreamSynchronize(stream_), "adjoint buffer reuse");
            if (d_padj_) cudaFree(d_padj_);
            d_padj_ = nullptr;
            check(cudaMalloc(&d_padj_, sizeof(float4) * words), "cudaMalloc(adjoint arrays)");
            padj_words_ = words;
        }
        if (!d_adj_args_) {
            check(cudaMalloc(&d_adj_args_, sizeof(FrameArgs)), "cudaMalloc(adjoint args)");
            check(cudaMallocHost(&h_adj_args_, sizeof(FrameArgs)), "cudaMallocHost(adjoint args)");
        }
        check(cudaStreamSynchronize(stream_), "adjoint args reuse");  // the previous backward read h_adj_args_
        *h_adj_args_ = a;
        check(cudaMemcpyAsync(d_adj_args_, h_adj_args_, sizeof(FrameArgs), cudaMemcpyHostToDevice, stream_), "upload(args)");
        const int surf = a.num_sdf > 0 ? 2 : (a.num_planes > 0 ? 1 : 0);
        check(launch_adjoint_plain(d_adj_args_, g, adjoint_plain_carve(d_padj_, n_, num_itr), n_, num_itr, substeps, surf,
                                   rope_contact_, rope_contact_ ? rope_grid() : nullptr, stream_),
              "adjoint (per launch)");
    } else {
        check(launch_adjoint(a, g, block_, (int)bins_.size(), stream_), "adjoint");
    }
    if (synchronize) check(cudaStreamSynchronize(stream_), "backward");
}

}  // namespace rs
