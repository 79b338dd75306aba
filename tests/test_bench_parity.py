"""Parity on the benchmarked scenes themselves: seeded samples of the ropes bench.py times,
replayed rope by rope through the FP64 oracle (and its FP32 instantiation).

The GPU steps the whole bench scene (config 2: 4096 x 64 ropes; config 3: 8192 uneven ropes with
two planes and eight moving meshes) for 60 control frames; the oracle steps only the sampled
ropes with the same inputs. That is exact because ropes never read each other without rope-rope
contact, and the product's result for a rope does not depend on which ropes share its CTA
(tests/test_gpu_parity.py::test_bitwise_replay_and_block_invariance).

Two comparisons, each against the FP64 oracle, with the FP32 oracle's deviation as the floor:
  * free run: both sides run 60 frames from the same start. The bound is 1e-5 m on every frame
    up to the one where the FP32 oracle itself first leaves 1e-5 m (the dynamics amplify
    rounding, so no FP32 run can follow FP64 further); after it, the GPU may deviate by at most
    4x the FP32 oracle's deviation + 1e-6 m.
  * re-synchronised: every frame both oracles start from the GPU's state at the frame start and
    run one frame. Each (rope, frame) case is bounded by 1e-5 m where the FP32 oracle stays within
    1e-5 m of FP64 on it, else by 4x the FP32 oracle's deviation + 1e-6 m; the counts are printed.

With RS_PARITY_OUT=<dir> the summary is also written there as parity_bench_scenes.json.
"""
import json
import os
import threading

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

TOL = 1e-5
FRAMES = 60
THREADS = max(1, min(16, os.cpu_count() or 1))


def _chunks(n):
    return [c for c in np.array_split(np.arange(n), min(n, THREADS)) if len(c)]


def _parallel(fn, items):
    out = [None] * len(items)

    def work(i):
        out[i] = fn(items[i])

    ts = [threading.Thread(target=work, args=(i,)) for i in range(len(items))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return out


def _rows(starts, ropes):
    return np.concatenate([np.arange(starts[r], starts[r + 1]) for r in ropes])


def _gpu_states(b, starts, sel, step, frames):
    """Caller-order (pos, vel, lvel, q) of the sampled ropes at the start and after every frame."""
    import ropesim.grad as rg

    idx = _rows(starts, sel)

    def grab():
        return tuple(t.cpu().numpy().astype(np.float64)[idx] for t in rg.state(b))

    out = [grab()]
    for f in range(frames):
        step(f)
        out.append(grab())
    return out


def _replay(build, step, sel, starts, gpu, precision):
    """Free-run and re-synchronised oracle positions of the sampled ropes: [F, n_sel_verts, 3] each."""
    loc = np.concatenate([[0], np.cumsum(np.diff(starts)[sel])])

    def chunk(c):
        ropes = sel[c]
        rows = np.concatenate([np.arange(loc[i], loc[i + 1]) for i in c])
        free, rs = build(ropes, precision), build(ropes, precision)
        # both runs start from the GPU's initial state (initial frames are transported along the
        # flat rope array, so a sample's first rope would otherwise start from another predecessor)
        st = free._s.get_state()
        g = gpu[0]
        free._s.set_state(g[0][rows], g[1][rows], g[2][rows], g[3][rows], st[4], st[5])
        fp, rp = [], []
        for f in range(FRAMES):
            st = rs._s.get_state()
            g = gpu[f]
            rs._s.set_state(g[0][rows], g[1][rows], g[2][rows], g[3][rows], st[4], st[5])
            step(free, ropes, f)
            step(rs, ropes, f)
            fp.append(np.asarray(free._s.positions(), np.float64))
            rp.append(np.asarray(rs._s.positions(), np.float64))
        return rows, np.stack(fp), np.stack(rp)

    n = int(loc[-1])
    free = np.zeros((FRAMES, n, 3))
    rs = np.zeros((FRAMES, n, 3))
    for rows, fp, rp in _parallel(chunk, _chunks(len(sel))):
        free[:, rows] = fp
        rs[:, rows] = rp
    return free, rs


def _per_rope(x, loc):
    """max over each rope's vertices: [F, n_verts] -> [F, n_ropes]"""
    return np.stack([x[:, loc[i]:loc[i + 1]].max(1) for i in range(len(loc) - 1)], 1)


def _judge(name, gpu, o64, o32, r64, r32, sel, starts):
    """Deviations per (frame, rope); the assertions of the module docstring; a summary dict."""
    loc = np.concatenate([[0], np.cumsum(np.diff(starts)[sel])])
    g = np.stack([s[0] for s in gpu[1:]])  # GPU positions after each frame
    d_free = _per_rope(np.linalg.norm(g - o64, axis=-1), loc)
    d_free32 = _per_rope(np.linalg.norm(o32 - o64, axis=-1), loc)
    d_rs = _per_rope(np.linalg.norm(g - r64, axis=-1), loc)
    d_rs32 = _per_rope(np.linalg.norm(r32 - r64, axis=-1), loc)
    # free run: frames before the FP32 oracle first leaves 1e-5 m, per rope
    within32 = np.maximum.accumulate(d_free32, axis=0) <= TOL
    strict_free = d_free[within32]
    floor_free = d_free.max(0) <= 4.0 * d_free32.max(0) + 1e-6
    # re-synchronised: per (frame, rope) case
    ok32 = d_rs32 <= TOL
    summary = {
        "ropes": int(len(sel)), "frames": FRAMES, "verts": int(loc[-1]),
        "free_run": {"gpu_vs_f64_max_m": float(d_free.max()), "f32_vs_f64_max_m": float(d_free32.max()),
                     "frames_within_1e-5_by_f32": int(within32.sum()),
                     "gpu_max_on_those_m": float(strict_free.max()) if strict_free.size else None,
                     "first_frame_gpu_vs_f64_m": float(d_free[0].max())},
        "resync": {"gpu_vs_f64_max_m": float(d_rs.max()), "f32_vs_f64_max_m": float(d_rs32.max()),
                   "gpu_vs_f64_median_m": float(np.median(d_rs)),
                   "cases": int(d_rs.size), "cases_held_to_1e-5": int(ok32.sum()),
                   "gpu_within_1e-5": int((d_rs <= TOL).sum()),
                   "gpu_max_on_held_cases_m": float(d_rs[ok32].max()) if ok32.any() else None,
                   "floor_cases_max_ratio": float((d_rs[~ok32] / (4.0 * d_rs32[~ok32] + 1e-6)).max()) if (~ok32).any() else None},
    }
    print(f"\n  {name}: {len(sel)} ropes ({loc[-1]} verts) x {FRAMES} frames")
    print(f"    free run : gpu-f64 max {d_free.max():.2e} m (f32-f64 {d_free32.max():.2e}); "
          f"{within32.sum()} rope-frames before f32 leaves 1e-5, gpu max there {summary['free_run']['gpu_max_on_those_m']}")
    print(f"    re-synced: gpu-f64 max {d_rs.max():.2e} m, median {np.median(d_rs):.2e} (f32-f64 max {d_rs32.max():.2e}); "
          f"{ok32.sum()} of {d_rs.size} cases held to 1e-5, gpu within 1e-5 in {(d_rs <= TOL).sum()}")
    out = os.environ.get("RS_PARITY_OUT")
    if out:
        path = os.path.join(out, "parity_bench_scenes.json")
        prev = json.load(open(path)) if os.path.exists(path) else {}
        prev[name] = summary
        json.dump(prev, open(path, "w"), indent=1)
    assert np.isfinite(g).all()
    assert strict_free.size == 0 or strict_free.max() <= TOL
    assert floor_free.all(), (d_free.max(0), d_free32.max(0))
    assert (d_rs[ok32] <= TOL).all(), d_rs[ok32].max()
    assert (d_rs[~ok32] <= 4.0 * d_rs32[~ok32] + 1e-6).all()
    return summary


def test_config2_bench_sample_parity():
    """32 of the bench's 4096 config-2 ropes (rank 0's seed), 60 frames of program driving."""
    import torch

    import ropesim
    import ropesim_oracle as ro

    N, V = 4096, 64
    pos, p0, v0, p1 = S.bench_c2_inputs(N, FRAMES, 1234)
    sel = np.sort(np.random.default_rng(2024).choice(N, 32, replace=False))
    starts = np.arange(N + 1) * V
    b = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, S.BENCH_H, S.BENCH_ITERS, deterministic=True)
    S.bench_c2_configure(b)
    P0, V0, P1 = (torch.as_tensor(x, device="cuda") for x in (p0, v0, p1))

    def gstep(f):
        b.step(P0[f], V0[f], S.BENCH_DT, S.BENCH_S, root_pos_end=P1[f])

    gpu = _gpu_states(b, starts, sel, gstep, FRAMES)

    def build(ropes, precision):
        o = ro.RopeBatch.from_positions(pos[ropes], 0.117, 11473.0, 4.48e-3, S.BENCH_H, S.BENCH_ITERS,
                                        deterministic=True, precision=precision)
        S.bench_c2_configure(o)
        return o

    def ostep(o, ropes, f):
        o.step(p0[f][ropes], v0[f][ropes], S.BENCH_DT, S.BENCH_S, root_pos_end=p1[f][ropes])

    o64, r64 = _replay(build, ostep, sel, starts, gpu, "f64")
    o32, r32 = _replay(build, ostep, sel, starts, gpu, "f32")
    _judge("config2", gpu, o64, o32, r64, r32, sel, starts)


def test_config3_bench_sample_parity():
    """48 of the bench's 8192 config-3 ropes, two per vertex-count band of width 10 over V = 16..256,
    60 frames with their own mesh poses (eight lattices, random rigid walks) and root programs."""
    import torch

    import ropesim
    import ropesim_oracle as ro
    from ropesim import sdf

    R = 8192
    scene = S.bench_c3_scene(sdf, R)
    verts = scene[1]
    PP, QQ, p0, v0, p1 = S.bench_c3_inputs(scene, FRAMES)
    rng = np.random.default_rng(2025)
    sel = []
    for lo in range(16, 257, 10):
        band = np.nonzero((verts >= lo) & (verts < lo + 10))[0]
        sel.extend(rng.choice(band, min(2, len(band)), replace=False).tolist())
    sel = np.sort(np.array(sel[:48]))
    starts = np.concatenate([[0], np.cumsum(verts)])
    b = S.bench_c3_build(ropesim, scene)
    T = [tuple(torch.as_tensor(x[f], device="cuda") for x in (PP, QQ, p0, v0, p1)) for f in range(FRAMES)]

    def gstep(f):
        b.set_mesh_poses_all(T[f][0], T[f][1], teleport=(f == 0))
        b.step(T[f][2], T[f][3], S.BENCH_DT, S.BENCH_S, root_pos_end=T[f][4])

    gpu = _gpu_states(b, starts, sel, gstep, FRAMES)
    del b, T

    def build(ropes, precision):
        return S.bench_c3_build(ro, scene, sel=ropes, precision=precision)

    def ostep(o, ropes, f):
        o.set_mesh_poses_all(PP[f][ropes], QQ[f][ropes], teleport=(f == 0))
        o.step(p0[f][ropes], v0[f][ropes], S.BENCH_DT, S.BENCH_S, root_pos_end=p1[f][ropes])

    o64, r64 = _replay(build, ostep, sel, starts, gpu, "f64")
    o32, r32 = _replay(build, ostep, sel, starts, gpu, "f32")
    _judge("config3", gpu, o64, o32, r64, r32, sel, starts)
