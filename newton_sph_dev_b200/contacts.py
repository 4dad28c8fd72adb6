"""Particle contacts: particle-particle contact on the HashGrid (the
reference's other grid consumers) and particle contact with static shapes,
on this library's kernels.

- :func:`eval_particle_contact_forces` replaces the launch of
  ``eval_particle_contact`` by SolverSemiImplicit
  (newton/_src/solvers/semi_implicit/kernels_contact.py:559-579).
- :func:`solve_particle_particle_contacts` replaces the launch of the XPBD
  kernel of the same name (newton/_src/solvers/xpbd/solver_xpbd.py:420-440).
- :func:`eval_particle_body_contact_forces`,
  :func:`solve_particle_shape_contacts`,
  :func:`apply_particle_shape_restitution` and :func:`apply_particle_deltas`
  replace the launches of eval_particle_body_contact (kernels_contact.py:
  644-690), solve_particle_shape_contacts (solver_xpbd.py:386-412),
  apply_particle_shape_restitution (solver_xpbd.py:686-714) and
  apply_particle_deltas (solver_xpbd.py:157-197) for shapes without a body.

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


def soft_contact_params(model, dt: float = 0.0, relaxation: float = 0.0) -> _lib.NsphSoftContactParams:
    return _lib.NsphSoftContactParams(float(model.soft_contact_ke), float(model.soft_contact_kd),
                                      float(model.soft_contact_kf), float(model.soft_contact_mu),
                                      float(model.particle_adhesion), float(model.soft_contact_restitution),
                                      float(relaxation), float(dt))


def _shapes_ptr(model) -> int:
    if model._shapes_dev is None:
        model.shapes_device()
    return model._shapes_dev.data_ptr()


def eval_particle_body_contact_forces(model, state, contacts, particle_f: torch.Tensor) -> None:
    """Subtract the particle-shape contact forces from particle_f (N, 3)
    (eval_particle_body_contact for static shapes). Does nothing without
    contacts or shapes."""
    if contacts is None or not contacts.soft_contact_max or not model.shape_count:
        return
    n = model.particle_count
    for t, name in ((state.particle_q, "particle_q"), (state.particle_qd, "particle_qd"), (particle_f, "particle_f")):
        _check(t, n, name)
    c = contacts.c_struct()
    p = soft_contact_params(model)
    st = _lib.load().nsph_particle_shape_contact_forces(
        _shapes_ptr(model), model.shape_count, ctypes.byref(c), ctypes.byref(p), state.particle_q.data_ptr(),
        state.particle_qd.data_ptr(), model.particle_radius.data_ptr(), model.particle_flags.data_ptr(),
        particle_f.data_ptr(), _lib.stream_handle(model.device))
    _lib.check(st, "eval_particle_body_contact_forces")


def solve_particle_shape_contacts(model, particle_q: torch.Tensor, particle_qd: torch.Tensor, contacts,
                                  particle_deltas: torch.Tensor, dt: float, relaxation: float) -> None:
    """Add the XPBD particle-shape contact corrections to particle_deltas."""
    if contacts is None or not contacts.soft_contact_max or not model.shape_count:
        return
    n = model.particle_count
    for t, name in ((particle_q, "particle_q"), (particle_qd, "particle_qd"), (particle_deltas, "particle_deltas")):
        _check(t, n, name)
    c = contacts.c_struct()
    p = soft_contact_params(model, dt, relaxation)
    st = _lib.load().nsph_particle_shape_contact_deltas(
        _shapes_ptr(model), model.shape_count, ctypes.byref(c), ctypes.byref(p), particle_q.data_ptr(),
        particle_qd.data_ptr(), model.particle_inv_mass.data_ptr(), model.particle_radius.data_ptr(),
        model.particle_flags.data_ptr(), particle_deltas.data_ptr(), _lib.stream_handle(model.device))
    _lib.check(st, "solve_particle_shape_contacts")


def apply_particle_shape_restitution(model, contacts, v_new: torch.Tensor, x_old: torch.Tensor,
                                     v_old: torch.Tensor, v_out: torch.Tensor) -> None:
    """Add the restitution velocity change of every approaching contact to v_out."""
    if contacts is None or not contacts.soft_contact_max:
        return
    c = contacts.c_struct()
    p = soft_contact_params(model)
    st = _lib.load().nsph_particle_shape_restitution(
        ctypes.byref(c), ctypes.byref(p), v_new.data_ptr(), x_old.data_ptr(), v_old.data_ptr(),
        model.particle_radius.data_ptr(), model.particle_flags.data_ptr(), v_out.data_ptr(),
        _lib.stream_handle(model.device))
    _lib.check(st, "apply_particle_shape_restitution")


def apply_particle_deltas(model, x_orig: torch.Tensor, x_pred: torch.Tensor, deltas: torch.Tensor, dt: float,
                          x_out: torch.Tensor, v_out: torch.Tensor) -> None:
    """x_out = x_pred + deltas, v_out = (x_out - x_orig)/dt clamped to
    model.particle_max_velocity, for active particles."""
    n = model.particle_count
    st = _lib.load().nsph_apply_particle_deltas(
        n, x_orig.data_ptr(), x_pred.data_ptr(), model.particle_flags.data_ptr(), deltas.data_ptr(), float(dt),
        float(model.particle_max_velocity), x_out.data_ptr(), v_out.data_ptr(), _lib.stream_handle(model.device))
    _lib.check(st, "apply_particle_deltas")


__all__ = ["apply_particle_deltas", "apply_particle_shape_restitution", "contact_params",
           "eval_particle_body_contact_forces", "eval_particle_contact_forces", "soft_contact_params",
           "solve_particle_particle_contacts", "solve_particle_shape_contacts"]
