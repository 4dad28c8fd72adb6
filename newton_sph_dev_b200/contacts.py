"""Particle-particle contact on the HashGrid: the reference's other grid
consumers, on this library's grid and kernels.

- :func:`eval_particle_contact_forces` replaces the launch of
  ``eval_particle_contact`` by SolverSemiImplicit
  (newton/_src/solvers/semi_implicit/kernels_contact.py:559-579).
- :func:`solve_particle_particle_contacts` replaces the launch of the XPBD
  kernel of the same name (newton/_src/solvers/xpbd/solver_xpbd.py:420-440).

Both read ``model.particle_grid`` (a :class:`HashGrid` built on the positions
they are given, with a cell width covering r_i + max_radius + cohesion, as
``model.particle_grid.build(q, 2 * model.particle_max_radius +
model.particle_cohesion)`` does) and the model's contact coefficients.
Stream-ordered on the current torch stream, no allocation.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


def _grid_ready(model) -> bool:
    grid = getattr(model, "particle_grid", None)
    return model.particle_count > 1 and grid is not None and grid.num_points == model.particle_count


def _check(t, n, name, width=3):
    shape = (n, width) if width else (n,)
    if t.dtype != (torch.int32 if name == "flags" else torch.float32) or tuple(t.shape) != shape or \
            not t.is_contiguous() or not t.is_cuda:
        raise ValueError(f"{name} must be a contiguous CUDA tensor of shape {shape}")


def contact_params(model) -> _lib.NsphContactParams:
    return _lib.NsphContactParams(float(model.particle_ke), float(model.particle_kd), float(model.particle_kf),
                                  float(model.particle_mu), float(model.particle_cohesion),
                                  float(model.particle_max_radius))


def eval_particle_contact_forces(model, state, particle_f: torch.Tensor) -> None:
    """Write the particle-particle contact force of every active particle
    into particle_f (N, 3); other rows are left as they are. Does nothing
    when the model has fewer than two particles, no grid, or a grid not yet
    built on these particles (as the reference's kernel returns early)."""
    if not _grid_ready(model):
        return
    n = model.particle_count
    for t, name in ((state.particle_q, "particle_q"), (state.particle_qd, "particle_qd"), (particle_f, "particle_f")):
        _check(t, n, name)
    _check(model.particle_radius, n, "particle_radius", 0)
    _check(model.particle_flags, n, "flags", 0)
    p = contact_params(model)
    L = _lib.load()
    st = L.nsph_particle_contact_forces(model.particle_grid.id, ctypes.byref(p), n, state.particle_q.data_ptr(),
                                        state.particle_qd.data_ptr(), model.particle_radius.data_ptr(),
                                        model.particle_flags.data_ptr(), particle_f.data_ptr(),
                                        _lib.stream_handle(model.device))
    _lib.check(st, "eval_particle_contact_forces")


def solve_particle_particle_contacts(model, particle_q: torch.Tensor, particle_qd: torch.Tensor,
                                     particle_deltas: torch.Tensor, dt: float, relaxation: float) -> None:
    """Add the XPBD particle-particle contact correction of every active
    particle to particle_deltas (N, 3)."""
    if not _grid_ready(model) or not (model.particle_max_radius > 0.0):
        return
    n = model.particle_count
    for t, name in ((particle_q, "particle_q"), (particle_qd, "particle_qd"), (particle_deltas, "particle_deltas")):
        _check(t, n, name)
    L = _lib.load()
    st = L.nsph_particle_contact_deltas(model.particle_grid.id, n, particle_q.data_ptr(), particle_qd.data_ptr(),
                                        model.particle_inv_mass.data_ptr(), model.particle_radius.data_ptr(),
                                        model.particle_flags.data_ptr(), float(model.particle_mu),
                                        float(model.particle_cohesion), float(model.particle_max_radius), float(dt),
                                        float(relaxation), particle_deltas.data_ptr(),
                                        _lib.stream_handle(model.device))
    _lib.check(st, "solve_particle_particle_contacts")


__all__ = ["contact_params", "eval_particle_contact_forces", "solve_particle_particle_contacts"]
