"""Generate the golden fixtures of tests/golden/ from the FP64 CPU oracle.

The reference ships no golden vectors (its tests are analytic), so these fixtures freeze the
oracle's FP64 trajectories of the well-posed parity scenes after the oracle passed the
reference's known-answer checks (tests/test_physics.py). They guard the oracle against silent
drift (CPU test) and give the GPU product a stored target (GPU test).

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import ropesim_oracle  # noqa: E402
import scenarios as S  # noqa: E402


def host(a):
    return np.asarray(a, np.float32)


def main():
    c1 = S.c1(ropesim_oracle, precision="f64")
    np.savez_compressed(os.path.join(HERE, "c1_f64.npz"), positions=c1)
    prog = S.program(ropesim_oracle, to_dev=host, precision="f64", v_std=0.05, p_std=0.005, N=4, frames=10)
    np.savez_compressed(os.path.join(HERE, "program_gentle_f64.npz"), positions=prog)
    leg = S.legacy(ropesim_oracle, to_dev=host, precision="f64", frames=15)
    np.savez_compressed(os.path.join(HERE, "legacy_f64.npz"), positions=leg)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
