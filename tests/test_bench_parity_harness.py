"""The bench-parity replay (tests/test_bench_parity.py) checked on the CPU: an FP64 oracle run of a
whole (reduced) bench scene stands in for the GPU, and the sampled replay, which rebuilds only a
few ropes and imports the scene's state into them, must reproduce that run to rounding.

This pins the harness itself: the state import (positions, velocities, last velocities,
rotors) and the per-rope frame-gauge mapping (initial frames are transported along the whole flat
rope array, so a sample's frames differ from the scene's by one twist per rope)."""
import numpy as np

import scenarios as S
import test_bench_parity as T

FRAMES = 3


def _scene_states(o, idx, step):
    out = []

    def grab():
        st = o._s.get_state()
        return tuple(np.asarray(st[k], np.float64)[idx] for k in range(4))

    out.append(grab())
    for f in range(FRAMES):
        step(f)
        out.append(grab())
    return out


def _check(gpu, free, rs):
    g = np.stack([s[0] for s in gpu[1:]])
    assert np.abs(free - g).max() < 1e-9, np.abs(free - g).max()
    assert np.abs(rs - g).max() < 1e-9, np.abs(rs - g).max()


def test_replay_reproduces_a_scene_run_config2():
    import ropesim_oracle as ro

    N, V = 48, 64
    pos, p0, v0, p1 = S.bench_c2_inputs(N, FRAMES, 1234)
    sel = np.array([3, 17, 30, 47])
    starts = np.arange(N + 1) * V
    o = ro.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, S.BENCH_H, S.BENCH_ITERS, deterministic=True,
                                    precision="f64")
    S.bench_c2_configure(o)
    gpu = _scene_states(o, T._rows(starts, sel),
                        lambda f: o.step(p0[f], v0[f], S.BENCH_DT, 20, root_pos_end=p1[f]))

    def build(ropes, precision):
        b = ro.RopeBatch.from_positions(pos[ropes], 0.117, 11473.0, 4.48e-3, S.BENCH_H, S.BENCH_ITERS,
                                        deterministic=True, precision=precision)
        S.bench_c2_configure(b)
        return b

    def ostep(b, ropes, f):
        b.step(p0[f][ropes], v0[f][ropes], S.BENCH_DT, 20, root_pos_end=p1[f][ropes])

    # the frames really are gauged differently in the sample (else the mapping is untested)
    q_sample = np.asarray(build(sel, "f64")._s.get_state()[3], np.float64)
    assert np.abs(q_sample - gpu[0][3]).max() > 1e-3
    free, rs = T._replay(build, ostep, sel, starts, gpu, "f64", frames=FRAMES)
    _check(gpu, free, rs)


def test_replay_reproduces_a_scene_run_config3():
    import ropesim_oracle as ro
    from ropesim import sdf

    R = 24
    scene = S.bench_c3_scene(sdf, R)
    verts = scene[1]
    PP, QQ, p0, v0, p1 = S.bench_c3_inputs(scene, FRAMES)
    sel = np.array([2, 9, 15, 23])
    starts = np.concatenate([[0], np.cumsum(verts)])
    o = S.bench_c3_build(ro, scene, precision="f64")

    def sstep(f):
        o.set_mesh_poses_all(PP[f], QQ[f], teleport=(f == 0))
        o.step(p0[f], v0[f], S.BENCH_DT, 20, root_pos_end=p1[f])

    gpu = _scene_states(o, T._rows(starts, sel), sstep)

    def build(ropes, precision):
        return S.bench_c3_build(ro, scene, sel=ropes, precision=precision)

    def ostep(b, ropes, f):
        b.set_mesh_poses_all(PP[f][ropes], QQ[f][ropes], teleport=(f == 0))
        b.step(p0[f][ropes], v0[f][ropes], S.BENCH_DT, 20, root_pos_end=p1[f][ropes])

    free, rs = T._replay(build, ostep, sel, starts, gpu, "f64", frames=FRAMES)
    _check(gpu, free, rs)
