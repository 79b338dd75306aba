"""Backend plumbing for the acceptance suites (test infrastructure).

"oracle" is the FP64 CPU restatement (host numpy inputs), "cuda" the product (ropesim, inputs
as float32 CUDA tensors, outputs read back from the device views). Both expose the ropesim API,
so one test body checks the oracle on the CPU and the product on the GPU.
"""
from __future__ import annotations

import numpy as np


def module(backend):
    if backend == "oracle":
        import ropesim_oracle

        return ropesim_oracle
    import ropesim

    return ropesim


def dev(backend, a, dtype=np.float32):
    """A step / pose input: numpy for the oracle, a CUDA tensor for the product."""
    a = np.ascontiguousarray(np.asarray(a, dtype))
    if backend == "oracle":
        return a
    import torch

    return torch.as_tensor(a, device="cuda")


def host(a):
    """Positions / velocities / frames / readouts of either backend as float64 numpy."""
    if hasattr(a, "__cuda_array_interface__"):
        import torch

        return torch.as_tensor(a).cpu().numpy().astype(np.float64)
    return np.asarray(a, np.float64)


def P(b):
    return host(b.positions())


def Vel(b):
    return host(b.velocities())


def Q(b):
    return host(b.quaternions())
