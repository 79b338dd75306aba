"""Count the algorithmic FLOPs per vertex-substep of the config-2 workload with the oracle's
op-counting scalar (TEST / MEASUREMENT INFRASTRUCTURE). Writes profiles/flop_count_config2.txt,
which bench.py reads for the roofline's `achieved` figure.

Counted: add/sub, mul, div, sqrt and transcendental calls of the restated substep (root
program, inertial prediction, num_itr position + frame steps, plane contact, velocity update),
for the workload's own inputs: 64-vertex jittered ropes, root program with v0 ~ N(0, 0.5) m/s,
p1 = p0 + N(0, 0.05) m, plane z = 0 at radius 6.35 mm, h = 1/6000, 8 iterations, 100 substeps.

Usage: python oracle/count_flops.py [ropes] [frames]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(ROOT, "tests")]


def count(ropes=16, frames=3, seed=0):
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
    flops = d["add"] + d["mul"] + d["div"] + d["sqrt"] + d["trans"]
    return flops / vs, {k: v / vs for k, v in d.items()}


def main():
    ropes = int(sys.argv[1]) if len(sys.argv) > 1 else 16
    frames = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    per, parts = count(ropes, frames)
    out = os.path.join(ROOT, "profiles", "flop_count_config2.txt")
    with open(out, "w") as f:
        f.write("# Algorithmic FP32 operations per vertex-substep, config-2 workload (4096 x 64, 100 substeps, 8 itr).\n")
        f.write(f"# command: python oracle/count_flops.py {ropes} {frames}\n")
        f.write("# counted by rso::Sim<OpCount> (oracle/rs_opcount.hpp) over the restated substep;\n")
        f.write("# add/sub, mul, div, sqrt, transcendental each = 1 FLOP; comparisons/min/max not counted.\n")
        for k, v in parts.items():
            f.write(f"{k}_per_vertex_substep: {v:.3f}\n")
        f.write(f"flops_per_vertex_substep: {per:.3f}\n")
    print(open(out).read())


if __name__ == "__main__":
    main()
