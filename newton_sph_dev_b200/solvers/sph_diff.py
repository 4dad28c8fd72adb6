"""Differentiable SPH steps and rollouts for torch.autograd.

The reference differentiates a simulation with ``wp.Tape``: the forward steps
run under the tape, every intermediate array is kept, and
``tape.backward(loss)`` replays Warp's generated adjoint kernels in reverse
(newton/solvers.py:359-395; examples/diffsim/example_diffsim_ball.py:
115-151). Here the adjoint of a step is hand-written CUDA
(``nsph_sph_step_adjoint``) and autograd sees it through two functions:

- :func:`sph_step` — one step as an autograd node. Like the tape, a loop of
  them keeps every state; any torch code may sit between steps.
- :func:`sph_rollout` — ``steps`` steps as one node with checkpointing: the
  forward keeps only every ``checkpoint_every``-th state, and the backward
  recomputes each segment from its checkpoint before reversing it
  (``nsph_sph_segment_adjoint``, which keeps each recomputed step's grid,
  density scratch and force sums so that the reverse does not recompute
  them), so memory is
  O(N (steps / K + K)) instead of O(N steps). The forward step is
  deterministic, so the recomputed states are bit-identical to the first
  pass.

Differentiable inputs: initial positions and velocities, the EOS stiffness
B (a one-element tensor) and a constant external force. The neighbour set is
held fixed within a step (the cubic spline and its derivative vanish at
r = h, so the step is C1 where it changes); clamps and walls are
differentiated on the side the forward took. The functions read B to the
host (a synchronisation), so they are not for use inside a CUDA graph
capture.
"""

from __future__ import annotations

import torch

from .sph import SolverSPH


def _b_value(solver: SolverSPH, eos_b) -> float:
    if eos_b is None:
        return float(solver.params_for(0.0).eos_b)
    return float(eos_b.detach().reshape(-1)[0].item()) if torch.is_tensor(eos_b) else float(eos_b)


def _forward_step(solver, x, v, params, f_ext):
    x1 = torch.empty_like(x)
    v1 = v.clone()  # inactive particles keep their velocity
    solver.step_raw(x, v, x1, v1, params, f_ext)
    return x1, v1


class _SPHStep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, eos_b, f_ext, solver, dt):
        x, v = x.detach().contiguous(), v.detach().contiguous()
        f = f_ext.detach().contiguous() if f_ext is not None else None
        params = solver.step_params(dt, _b_value(solver, eos_b))
        x1, v1 = _forward_step(solver, x, v, params, f)
        ctx.solver, ctx.params = solver, params
        ctx.has_b, ctx.has_f = torch.is_tensor(eos_b), f_ext is not None
        ctx.b_meta = (eos_b.dtype, eos_b.shape) if torch.is_tensor(eos_b) else None
        ctx.save_for_backward(x, v, f if f is not None else torch.empty(0, device=x.device))
        return x1, v1

    @staticmethod
    def backward(ctx, gx, gv):
        x, v, f = ctx.saved_tensors
        f = f if ctx.has_f else None
        solver = ctx.solver
        gx = torch.zeros_like(x) if gx is None else gx.contiguous().float()
        gv = torch.zeros_like(v) if gv is None else gv.contiguous().float()
        xg, vg = torch.empty_like(x), torch.empty_like(v)
        bg = torch.zeros(1, dtype=torch.float32, device=x.device)
        fg = torch.zeros_like(x) if f is not None else None
        solver.step_backward_raw(x, v, ctx.params, gx, gv, xg, vg, f_ext=f, f_ext_grad=fg, eos_b_grad=bg)
        gb = bg.to(ctx.b_meta[0]).reshape(ctx.b_meta[1]) if ctx.has_b else None
        return xg, vg, gb, fg, None, None


def sph_step(solver: SolverSPH, x: torch.Tensor, v: torch.Tensor, dt: float, eos_b: torch.Tensor | None = None,
             f_ext: torch.Tensor | None = None) -> tuple[torch.Tensor, torch.Tensor]:
    """One differentiable WCSPH step (x, v) -> (x1, v1) of `solver`'s model.

    Args:
        x, v: (N, 3) float32 CUDA tensors.
        dt: time step [s].
        eos_b: EOS stiffness B as a one-element tensor (to get its gradient)
            or None for the solver config's value.
        f_ext: constant (N, 3) external force or None.
    """
    return _SPHStep.apply(x, v, eos_b, f_ext, solver, float(dt))


class _SPHRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, eos_b, f_ext, solver, steps, dt, every):
        x = x0.detach().contiguous().clone()  # the first checkpoint
        v = v0.detach().contiguous().clone()
        n = x.shape[0]
        f = f_ext.detach().contiguous() if f_ext is not None else None
        params = solver.step_params(dt, _b_value(solver, eos_b))
        tx = torch.empty((min(every, steps), n, 3), dtype=torch.float32, device=x.device)
        tv = torch.empty_like(tx)
        checkpoints = []
        for start, length in reversed(checkpoint_schedule(steps, every)):
            checkpoints.append((x, v))
            solver.rollout_raw(x, v, tx[:length], tv[:length], params, f)
            x, v = tx[length - 1].clone(), tv[length - 1].clone()
        ctx.solver, ctx.params, ctx.steps, ctx.every = solver, params, steps, every
        ctx.checkpoints = checkpoints
        ctx.f = f
        ctx.has_b = torch.is_tensor(eos_b)
        ctx.b_meta = (eos_b.dtype, eos_b.shape) if ctx.has_b else None
        return x, v

    @staticmethod
    def backward(ctx, gx, gv):
        solver, params, steps, every, f = ctx.solver, ctx.params, ctx.steps, ctx.every, ctx.f
        x0 = ctx.checkpoints[0][0]
        n = x0.shape[0]
        xa = torch.zeros_like(x0) if gx is None else gx.contiguous().float().clone()
        va = torch.zeros_like(x0) if gv is None else gv.contiguous().float().clone()
        bg = torch.zeros(1, dtype=torch.float32, device=x0.device)
        fg = torch.zeros_like(x0) if f is not None else None
        for c, (start, length) in enumerate(checkpoint_schedule(steps, every)):
            # recompute the segment from its checkpoint, keeping each step's
            # grid and density scratch, and reverse it
            cx, cv = ctx.checkpoints[len(ctx.checkpoints) - 1 - c]
            solver.segment_backward_raw(cx, cv, length, params, xa, va, f_ext=f, f_ext_grad=fg, eos_b_grad=bg)
        ctx.checkpoints = None
        gb = bg.to(ctx.b_meta[0]).reshape(ctx.b_meta[1]) if ctx.has_b else None
        return xa, va, gb, fg, None, None, None, None


def sph_rollout(solver: SolverSPH, x0: torch.Tensor, v0: torch.Tensor, steps: int, dt: float,
                eos_b: torch.Tensor | None = None, f_ext: torch.Tensor | None = None,
                checkpoint_every: int = 10) -> tuple[torch.Tensor, torch.Tensor]:
    """`steps` differentiable WCSPH steps from (x0, v0), checkpointed.

    The backward pass costs one extra forward step per step (the segment
    recompute, whose grid build, density pass and force sums the adjoint
    step then reuses) plus the adjoint step, and holds steps /
    checkpoint_every checkpoints plus one segment's tape (120 bytes per
    particle and 8 per grid cell, per step).

    Returns:
        (x_T, v_T), each (N, 3) float32.
    """
    steps, every = int(steps), int(checkpoint_every)
    if steps < 0 or every < 1:
        raise ValueError("steps must be >= 0 and checkpoint_every >= 1")
    if steps == 0:
        return x0, v0
    return _SPHRollout.apply(x0, v0, eos_b, f_ext, solver, steps, float(dt), every)


def checkpoint_schedule(steps: int, every: int) -> list[tuple[int, int]]:
    """(start, length) of the checkpointed segments of a rollout, in the
    order the backward pass reverses them."""
    if steps < 0 or every < 1:
        raise ValueError("steps must be >= 0 and checkpoint_every >= 1")
    segs = [(s, min(every, steps - s)) for s in range(0, steps, every)]
    return segs[::-1]


__all__ = ["sph_step", "sph_rollout", "checkpoint_schedule"]
