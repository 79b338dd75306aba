"""Differentiable control frames of a RopeBatch: torch.autograd over the CUDA adjoint.

The reference has no gradients; this module is new surface. One call of `frame` advances the
batch by one program-driven control frame (the same kernel as `RopeBatch.step(...,
root_pos_end=...)`) from an explicit state and explicit parameters, and its backward runs the
hand-written adjoint kernel (rs_batch_backward): the frame is replayed from its start state
(the per-frame checkpoint autograd keeps), each substep's start state is taped in HBM, and the
substeps are reversed with their iterates recomputed in shared memory.

    import ropesim, ropesim.grad as rg
    b = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8)
    state = rg.state(b)                               # (pos, vel, lvel, q): [n,3], [n,3], [n,3], [n,4]
    ea, ei, mass = (t.requires_grad_() for t in rg.parameters(b))   # [n] each
    for f in range(F):
        state = rg.frame(b, state, (ea, ei, mass), p0[f], v0[f], p1[f], 1 / 60, 100)
        loss = loss + ((state[0].view(R, V, 3)[:, -1] - target[f]) ** 2).mean()
    loss.backward()                                   # grads of ea, ei, mass, p0/v0/p1, the initial state

Arrays are float32 CUDA tensors in caller order (rope r's vertices consecutive). `lvel` is the
velocity at the last substep's start (the next substep's initial guess extrapolates from it).
EA / EI are per segment i -> i+1 (a rope's last vertex is ignored, its gradient is 0); mass is
per vertex (pinned vertices are ignored, gradient 0). Differentiated: root program, inertia,
gravity, linear and quadratic drag, damping, stretch, bending/twist frames and plane contact
with friction, through every iteration of the local solve; contact, friction regime and
frame-step signs are held where the forward pass took them. Rope-rope and mesh contact are
refused with ValueError.
"""
from __future__ import annotations

import torch

__all__ = ["state", "parameters", "frame", "Frame"]


def _n(batch):
    return int(batch.num_verts)


def _check(t, shape, name):
    if t is None:
        return None
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32):
        raise ValueError(f"{name} must be a float32 CUDA tensor")
    if tuple(t.shape) != tuple(shape):
        t = t.reshape(shape)
    # the engine reads raw device memory (torch hides __cuda_array_interface__ on tensors that
    # require grad); autograd sees the inputs through Frame itself
    return t.detach().contiguous()


def _ptr(t):
    return 0 if t is None else t.data_ptr()


def state(batch):
    """Copies of the batch's current (pos, vel, lvel, q) as [n,3], [n,3], [n,3], [n,4] tensors."""
    n = _n(batch)
    out = [torch.empty(n, k, device="cuda", dtype=torch.float32) for k in (3, 3, 3, 4)]
    batch.get_state(*out)
    return tuple(out)


def parameters(batch):
    """Copies of the batch's per-vertex (EA, EI, mass) as [n] tensors (0 where not applicable)."""
    n = _n(batch)
    out = [torch.empty(n, device="cuda", dtype=torch.float32) for _ in range(3)]
    batch.get_parameters(*out)
    return tuple(out)


class Frame(torch.autograd.Function):
    """(pos, vel, lvel, q, ea, ei, mass, p0, v0, p1) -> frame-end (pos, vel, lvel, q).

    Forward and backward are one library call each (rs_batch_frame_forward, rs_batch_backward),
    queued on the batch's stream without host synchronization; torch's current stream and the
    batch's stream are ordered with events on both sides."""

    @staticmethod
    def forward(ctx, batch, dt, substeps, tape, pos, vel, lvel, q, ea, ei, mass, p0, v0, p1):
        n, R = _n(batch), int(batch.num_envs)
        ctx.shapes = [None if t is None else tuple(t.shape) for t in (pos, vel, lvel, q, ea, ei, mass, p0, v0, p1)]
        ctx.free = p0 is None
        pos, vel, lvel = (_check(t, (n, 3), k) for t, k in ((pos, "pos"), (vel, "vel"), (lvel, "lvel")))
        q = _check(q, (n, 4), "q")
        ea, ei, mass = (_check(t, (n,), k) for t, k in ((ea, "ea"), (ei, "ei"), (mass, "mass")))
        if (p0 is None) != (v0 is None) or (p0 is None) != (p1 is None):
            raise ValueError("a program frame needs p0, v0 and p1 (all None: a free frame)")
        if p0 is not None:
            p0, v0, p1 = (_check(t, (R, 3), k) for t, k in ((p0, "p0"), (v0, "v0"), (p1, "p1")))
        out = [torch.empty(n, k, device="cuda", dtype=torch.float32) for k in (3, 3, 3, 4)]
        # the frame's substep tape (64 B per vertex-substep) lets the backward skip the replay;
        # the iterate tape (48 B per vertex-substep-iteration: d, q and the frame step's blend
        # rotor b) also skips the recomputation
        ctx.tape = torch.empty(16 * int(substeps) * n, device="cuda", dtype=torch.float32) if tape else None
        ctx.itape = None
        if tape == "iterates":
            ctx.itape = torch.empty(12 * int(batch.num_itr) * int(substeps) * n, device="cuda", dtype=torch.float32)
        cur, ext = _streams(batch)
        ext.wait_stream(cur)
        ptrs = [_ptr(t) for t in (pos, vel, lvel, q, ea, ei, mass, p0, v0, p1)] + [_ptr(t) for t in out]
        ptrs += [_ptr(ctx.tape), _ptr(ctx.itape)]
        last_h = batch._frame_forward(ptrs, float(dt), int(substeps))
        cur.wait_stream(ext)
        ctx.batch, ctx.dt, ctx.substeps, ctx.last_h = batch, float(dt), int(substeps), float(last_h)
        ctx.save_for_backward(pos, vel, lvel, q, ea, ei, mass, p0, v0, p1)
        return tuple(out)

    @staticmethod
    def backward(ctx, g_pos, g_vel, g_lvel, g_q):
        pos, vel, lvel, q, ea, ei, mass, p0, v0, p1 = ctx.saved_tensors
        b = ctx.batch
        n, R = pos.shape[0], int(b.num_envs)
        g_in = [None if g is None else g.detach().contiguous().to(torch.float32) for g in (g_pos, g_vel, g_lvel, g_q)]
        o = [torch.empty(n, 3, device="cuda", dtype=torch.float32) for _ in range(3)]
        o.append(torch.empty(n, 4, device="cuda", dtype=torch.float32))
        op = [torch.empty(n, device="cuda", dtype=torch.float32) for _ in range(3)]
        og = [None] * 3 if ctx.free else [torch.empty(R, 3, device="cuda", dtype=torch.float32) for _ in range(3)]
        ptrs = [_ptr(t) for t in (pos, vel, lvel, q, p0, v0, p1, None, None)]
        ptrs += [_ptr(t) for t in g_in] + [_ptr(t) for t in o] + [_ptr(t) for t in op] + [_ptr(t) for t in og]
        ptrs += [_ptr(ctx.tape), _ptr(ea), _ptr(ei), _ptr(mass), _ptr(ctx.itape)]
        cur, ext = _streams(b)
        ext.wait_stream(cur)
        b._backward(ptrs, ctx.dt, ctx.substeps, ctx.last_h)
        cur.wait_stream(ext)
        ctx.tape = ctx.itape = None
        grads = [None if t is None else t.reshape(sh) for t, sh in zip(o + op + og, ctx.shapes)]
        return (None, None, None, None, *grads)


def _streams(batch):
    cur = torch.cuda.current_stream()
    ext = getattr(batch, "_torch_stream", None)
    if ext is None:
        ext = torch.cuda.ExternalStream(batch.stream_ptr())
        try:
            batch._torch_stream = ext
        except AttributeError:
            pass
    return cur, ext


def frame(batch, st, params, p0, v0, p1, dt, substeps, tape=True):
    """One differentiable control frame: returns the frame-end (pos, vel, lvel, q). p0, v0, p1
    ([R, 3] root program rows) all None make a free frame (no root driving, as step_free).

    tape=True keeps the frame's substep tape in device memory until the backward (64 B per
    vertex-substep: 420 MB for 65,536 vertices x 100 substeps), so the backward does not replay
    the frame; tape="iterates" also keeps every iterate (48 B per vertex-substep-iteration: 2.5 GB
    more at that size and 8 iterations), so the backward does not recompute them either (used on
    the persistent engine without rope-rope contact; elsewhere the backward recomputes);
    tape=False keeps only the frame-start state and replays the frame in the backward."""
    pos, vel, lvel, q = st
    ea, ei, mass = params
    ins = (pos, vel, lvel, q, ea, ei, mass, p0, v0, p1)
    if tape not in (True, False, "iterates"):
        raise ValueError("tape must be True, False or 'iterates'")
    grad = torch.is_grad_enabled() and any(isinstance(t, torch.Tensor) and t.requires_grad for t in ins)
    keep = (tape if tape else False) if grad else False
    return Frame.apply(batch, dt, substeps, keep, *ins)
