"""Count the algorithmic FLOPs per vertex-substep of the benchmarked workloads with the oracle's
op-counting scalar (TEST / MEASUREMENT INFRASTRUCTURE). Writes profiles/flop_count_<workload>.txt,
which bench.py reads for the roofline's `achieved` figure.

Counted: add/sub, mul, div, sqrt and transcendental calls of the restated substep (root program,
mesh poses, inertial prediction, num_itr position + frame steps, plane and lattice contact,
velocity update, broad phase), i.e. the reference algorithm's work: every candidate lattice is
sampled, as the reference does (the product's exact early outs skip some of those samples).

  config2: 64-vertex jittered ropes, root program with v0 ~ N(0, 0.5) m/s, p1 = p0 + N(0, 0.05) m,
           plane z = 0 at radius 6.35 mm, h = 1/6000, 8 iterations, 100 substeps.
  config3: a sample of the bench's own 8192 uneven ropes (the ropes of tests/test_bench_parity.py),
           two planes, eight moving 64^3 lattices, their own poses and programs, frames
           [first, first + frames) of the bench's inputs (the bench times frames 5..24).

Usage: python oracle/count_flops.py config2 [ropes] [frames]
       python oracle/count_flops.py config3 [frames] [first]
"""
import os
import sys
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(ROOT, "tests"), os.path.join(ROOT, "cosserat-rod-solver-cuda_b200")]

KEYS = ("add", "mul", "div", "sqrt", "trans", "cmp")


def count_config2(ropes=16, frames=3, seed=0):
    import _oracle
    import scenarios as S

    pos, roots = S.c2_positions(ropes, 64, seed)
    rng = np.random.default_rng(seed + 1)
    p0 = np.empty((frames, ropes, 3), np.float32)
    v0 = rng.normal(0, 0.5, (frames, ropes, 3)).astype(np.float32)
    p1 = np.empty_like(p0)
    cur = roots.copy()
    for f in range(frames):
        p0[f] = cur
        p1[f] = cur + rng.normal(0, 0.05, (ropes, 3))
        cur = p1[f]
    d = _oracle.count_program_ops(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8, p0, v0, p1, 1 / 60, 100,
                                  np.array([[0, 0, 1, 0]], np.float32), 0.00635)
    vs = d.pop("vertex_substeps")
    return d, vs


def config3_sample(verts, n=48, seed=2025):
    """Two ropes per vertex-count band of width 10 over V = 16..256 (the parity tests' sample)."""
    rng = np.random.default_rng(seed)
    sel = []
    for lo in range(16, 257, 10):
        band = np.nonzero((verts >= lo) & (verts < lo + 10))[0]
        sel.extend(rng.choice(band, min(2, len(band)), replace=False).tolist())
    return np.sort(np.array(sel[:n]))


def count_config3(frames=4, first=5, threads=None):
    import _oracle
    import ropesim_oracle as ro
    import scenarios as S
    from ropesim import sdf

    scene = S.bench_c3_scene(sdf, 8192)
    PP, QQ, p0, v0, p1 = S.bench_c3_inputs(scene, first + frames)
    sel = config3_sample(scene[1])
    threads = threads or min(16, os.cpu_count() or 1)
    chunks = [c for c in np.array_split(sel, threads) if len(c)]
    out = [None] * len(chunks)

    def work(i):
        c = chunks[i]
        o = S.bench_c3_build(ro, scene, sel=c, precision="ops")
        for f in range(first + frames):
            if f == first:
                _oracle.op_tally_reset()
            o.set_mesh_poses_all(PP[f][c], QQ[f][c], teleport=(f == 0))
            o.step(p0[f][c], v0[f][c], S.BENCH_DT, S.BENCH_S, root_pos_end=p1[f][c])
        out[i] = _oracle.op_tally()

    ts = [threading.Thread(target=work, args=(i,)) for i in range(len(chunks))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    d = {k: sum(o[k] for o in out) for k in KEYS}
    vs = int(scene[1][sel].sum()) * S.BENCH_S * frames
    return d, vs


def main():
    which = sys.argv[1] if len(sys.argv) > 1 else "config2"
    if which == "config2":
        ropes = int(sys.argv[2]) if len(sys.argv) > 2 else 16
        frames = int(sys.argv[3]) if len(sys.argv) > 3 else 3
        d, vs = count_config2(ropes, frames)
        head = ("# Algorithmic FP32 operations per vertex-substep, config-2 workload (4096 x 64, 100 substeps, 8 itr).\n"
                f"# command: python oracle/count_flops.py config2 {ropes} {frames}\n")
    else:
        frames = int(sys.argv[2]) if len(sys.argv) > 2 else 4
        first = int(sys.argv[3]) if len(sys.argv) > 3 else 5
        d, vs = count_config3(frames, first)
        head = ("# Algorithmic FP32 operations per vertex-substep, config-3 workload (8192 uneven ropes, 2 planes,\n"
                "# 8 moving 64^3 lattices, 100 substeps, 8 itr), counted on 48 of its ropes (2 per vertex-count\n"
                f"# band of 10) over frames {first}..{first + frames - 1} of the bench's inputs.\n"
                f"# command: python oracle/count_flops.py config3 {frames} {first}\n")
    parts = {k: d[k] / vs for k in KEYS}
    per = sum(parts[k] for k in ("add", "mul", "div", "sqrt", "trans"))
    out = os.path.join(ROOT, "profiles", f"flop_count_{which}.txt")
    with open(out, "w") as f:
        f.write(head)
        f.write("# counted by rso::Sim<OpCount> (oracle/rs_opcount.hpp) over the restated substep;\n")
        f.write("# add/sub, mul, div, sqrt, transcendental each = 1 FLOP; comparisons/min/max not counted.\n")
        for k, v in parts.items():
            f.write(f"{k}_per_vertex_substep: {v:.3f}\n")
        f.write(f"flops_per_vertex_substep: {per:.3f}\n")
    print(open(out).read())


if __name__ == "__main__":
    main()
