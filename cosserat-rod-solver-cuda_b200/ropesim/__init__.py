"""ropesim (B200 engine) -- drop-in for the reference's `ropesim` package.

- RopeSim:   one rope with a host-driven root (advance(dt, substeps), set_root, host getters).
- RopeBatch: N ropes in one solver, roots driven from CUDA tensors (constant velocity or the
             second-order motion program with SLERPed frames), zero-copy device views of
             positions / velocities / frames, planes, SDF meshes with per-env kinematic poses,
             force and wrench readout. `RopeBatch.from_ropes` adds uneven rope lengths.
- CudaView:  a device buffer with __cuda_array_interface__ (torch.as_tensor shares it).
- ropesim.sdf: signed-distance lattices (closed forms and sampled functions).

Every control frame runs as ONE persistent sm_100a kernel launch (whole ropes per CTA, vertex
state resident on chip across all substeps). The CUDA extension is required: there is no CPU
fallback, and importing this package without the built extension raises ImportError.

Units: density = rho [kg/m], k_stretch = EA [N], k_bend = EI [N*m^2] (> 0).
"""
from . import sdf  # noqa: F401

try:
    from ._ropesim import CudaView, RopeBatch, RopeSim  # noqa: F401
except ImportError as e:  # pragma: no cover - exercised only on a broken install
    raise ImportError(
        "ropesim: the CUDA engine (_ropesim / libropesim_b200.so) is not built; run "
        "`python cosserat-rod-solver-cuda_b200/build.py` (needs nvcc). There is no CPU fallback."
    ) from e

__all__ = ["RopeSim", "RopeBatch", "CudaView", "sdf"]
