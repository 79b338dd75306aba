"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the FP64 oracle).

CPU: the oracle still reproduces them (guards the checker against drift).
GPU: the product lands within the parity bound of 1e-5 m on every frame.
"""
import os

import numpy as np
import pytest

import scenarios as S

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))["positions"]


def host(a):
    return np.asarray(a, np.float32)


CASES = {
    "c1_f64.npz": lambda mod, to_dev, **kw: S.c1(mod, **kw),
    "program_gentle_f64.npz": lambda mod, to_dev, **kw: S.program(mod, to_dev=to_dev, v_std=0.05, p_std=0.005, N=4,
                                                                  frames=10, **kw),
    "legacy_f64.npz": lambda mod, to_dev, **kw: S.legacy(mod, to_dev=to_dev, frames=15, **kw),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    import ropesim_oracle

    out = CASES[name](ropesim_oracle, host, precision="f64")
    np.testing.assert_allclose(out, load(name), rtol=0, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_product_matches_golden(name):
    import torch

    import ropesim

    def to_dev(a):
        return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")

    if name.startswith("program"):
        out = S.program(ropesim, to_dev=to_dev, v_std=0.05, p_std=0.005, N=4, frames=10,
                        views=lambda b: torch.as_tensor(b.positions()).cpu().numpy().astype(np.float64))
    else:
        out = CASES[name](ropesim, to_dev)
    d = np.max(np.linalg.norm(out.reshape(load(name).shape) - load(name), axis=-1))
    print(f"\n  {name}: max deviation {d:.2e} m")
    assert d <= 1e-5
