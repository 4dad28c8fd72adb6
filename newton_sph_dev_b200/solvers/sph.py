"""SolverSPH: weakly-compressible SPH behind Newton's solver interface.

The reference (NVIDIA Newton) has no SPH solver. This solver keeps its
interface — ``SolverBase.step(state_in, state_out, control, contacts, dt)``
(newton/_src/solvers/solver.py:301-316), ``notify_model_changed``
(:318-345), ``register_custom_attributes`` (:358-366), a nested ``Config``
like ``SolverImplicitMPM.Config`` (solver_implicit_mpm.py:643) — and the
structure of its particle hot path: a HashGrid build on the particle
positions (solver_xpbd.py:315-319), per-particle neighbour gathers through
the grid (kernels_contact.py:35-84) and integrate_particles semantics
(solver.py:10-47).

One step = one ``nsph_sph_step`` call into libnsph.so: grid build (cell
counts, a single-pass scan of the cell table, stable ranking within each
cell and the sorted gather; the LSD radix sort for sparse cell tables),
density/EOS pass (neighbour lists), pressure/XSPH/integrate pass. Stream-ordered on the current torch stream,
no allocation and no host sync, so a step (or a loop of steps) can be
captured with ``torch.cuda.graph``. Gravity is read from ``model.gravity``
on the device, so ``model.set_gravity`` reaches replayed graphs; scalar
parameters (dt, h, ...) are kernel arguments and are frozen into a captured
graph, as they are in Warp.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib
from ..sim import Model, ModelBuilder, State
from ..sim.control import Control
from .flags import SolverNotifyFlags
from .solver import SolverBase, _require_cuda

F32 = np.float32


def _next_pow2(v: int) -> int:
    p = 1
    while p < v:
        p <<= 1
    return p


def _trunc(v: float) -> int:
    return int(math.trunc(v)) if math.isfinite(v) else 0


@dataclass
class SPHConfig:
    """Parameters of :class:`SolverSPH`.

    Attributes:
        smoothing_length: kernel support radius h [m] (the neighbour radius;
            the cubic spline vanishes at r = h). With h = 2 x spacing a
            particle has about 33 neighbours.
        rest_density: rho0 [kg/m^3].
        sound_speed: c0 [m/s] of the Tait equation of state.
        eos_gamma: Tait exponent (integer).
        xsph: XSPH velocity-smoothing coefficient epsilon.
        clamp_pressure: clamp negative pressure to 0 (no tensile suction at
            free surfaces and walls).
        box_lo, box_hi: axis-aligned domain [m]; dynamic particles are
            clamped to it and lose the velocity component into the wall.
            None disables the box.
        cell_width: grid cell width [m]; defaults to h.
        grid_dims: cells per axis of the neighbour grid; by default the
            smallest powers of two that cover the box plus one guard cell on
            each side (so no two box cells alias), else 128^3.
        apply_particle_f: add ``state_in.particle_f * inv_mass`` (external
            forces) to the acceleration, as integrate_particles does.
        arithmetic: "exact" (default: every fp32 operation of the density
            and force terms correctly rounded in the oracle's order, results
            bit-exact with the fp32 oracle) or "fast" (hardware reciprocal
            square root in the kernel terms; the same neighbour sets and
            summation order, results within the fp64 oracle's tolerance).
            Applies to the plain single-world step.
    """

    smoothing_length: float = 0.02
    rest_density: float = 1000.0
    sound_speed: float = 20.0
    eos_gamma: int = 7
    xsph: float = 0.01
    clamp_pressure: bool = True
    box_lo: tuple[float, float, float] | None = None
    box_hi: tuple[float, float, float] | None = None
    cell_width: float | None = None
    grid_dims: tuple[int, int, int] | None = None
    apply_particle_f: bool = True
    arithmetic: str = "exact"

    # ---- derived constants ------------------------------------------
    def constants(self, dt: float, v_max: float) -> dict:
        """fp32 constants handed to the device (and to the fp32 oracle), plus
        their fp64 counterparts for the fp64 oracle. The fp64 values start
        from the fp32-rounded h so both describe the same kernel support."""
        h32 = F32(self.smoothing_length)
        cw32 = F32(self.cell_width if self.cell_width is not None else self.smoothing_length)
        h = float(h32)
        sigma = 8.0 / (math.pi * h**3)
        b = self.rest_density * self.sound_speed**2 / self.eos_gamma if self.eos_gamma > 0 else 0.0
        use_box = self.box_lo is not None and self.box_hi is not None
        lo = tuple(float(F32(v)) for v in (self.box_lo if use_box else (0.0, 0.0, 0.0)))
        hi = tuple(float(F32(v)) for v in (self.box_hi if use_box else (0.0, 0.0, 0.0)))
        f32 = {
            "h": h32,
            "h2": F32(h32 * h32),
            "inv_h": F32(F32(1.0) / h32),
            "cell_width": cw32,
            "cell_inv": F32(F32(1.0) / cw32),
            "sigma": F32(sigma),
            "dsigma": F32(sigma / h),
            "c_near": F32(6.0 * sigma / (h * h)),
            "c_far": F32(-6.0 * sigma / h),
            "rho0": F32(self.rest_density),
            "inv_rho0": F32(1.0 / self.rest_density),
            "eos_b": F32(b),
            "eos_gamma": int(self.eos_gamma),
            "clamp_pressure": int(bool(self.clamp_pressure)),
            "xsph_eps": F32(self.xsph),
            "v_max": F32(v_max),
            "dt": F32(dt),
            "use_box": int(use_box),
            "box_lo": tuple(F32(v) for v in lo),
            "box_hi": tuple(F32(v) for v in hi),
        }
        f64 = {
            "h": h,
            "inv_h": 1.0 / h,
            "sigma": sigma,
            "dsigma": sigma / h,
            "c_near": 6.0 * sigma / (h * h),
            "c_far": -6.0 * sigma / h,
            "rho0": float(self.rest_density),
            "inv_rho0": 1.0 / self.rest_density,
            "eos_b": b,
            "xsph_eps": float(self.xsph),
            "v_max": float(v_max),
            "dt": float(dt),
            "box_lo": lo,
            "box_hi": hi,
            "eos_gamma": int(self.eos_gamma),
            "clamp_pressure": int(bool(self.clamp_pressure)),
            "use_box": int(use_box),
        }
        return {"f32": f32, "f64": f64}

    def resolved_grid_dims(self, tight: bool = False) -> tuple[int, int, int]:
        """Grid dims: `grid_dims` if given; else, with a box, the cells that
        cover it plus one guard cell per side, rounded up to powers of two
        (or exact when `tight`, as the batched-worlds grids use); else 128^3
        (64^3 when tight)."""
        if self.grid_dims is not None:
            return tuple(int(d) for d in self.grid_dims)
        if self.box_lo is None or self.box_hi is None:
            return (64, 64, 64) if tight else (128, 128, 128)
        inv = float(F32(1.0) / F32(self.cell_width if self.cell_width is not None else self.smoothing_length))
        dims = []
        for a in range(3):
            lo = _trunc(float(F32(F32(self.box_lo[a]) * F32(inv))))
            hi = _trunc(float(F32(F32(self.box_hi[a]) * F32(inv))))
            span = max(4, hi - lo + 3)
            dims.append(min(2048, span if tight else _next_pow2(span)))
        while dims[0] * dims[1] * dims[2] > (1 << 26):
            k = int(np.argmax(dims))
            dims[k] //= 2
        return tuple(dims)

    def params(self, dt: float, v_max: float) -> _lib.NsphSphParams:
        c = self.constants(dt, v_max)["f32"]
        p = _lib.NsphSphParams()
        for name, _ in _lib.NsphSphParams._fields_:
            val = c[name]
            if name in ("box_lo", "box_hi"):
                getattr(p, name)[:] = [float(v) for v in val]
            elif isinstance(val, int):
                setattr(p, name, val)
            else:
                setattr(p, name, float(val))
        return p


class SolverSPH(SolverBase):
    """WCSPH particle-fluid solver on one CUDA device.

    With one ``Config`` every particle shares one grid and one parameter set
    (particles of different worlds interact, as in the reference's particle
    kernels, which ignore ``particle_world``). With a list of configs, one
    per world (``model.world_count`` entries), the solver runs in
    batched-worlds mode: each world has its own grid and parameters, a
    particle only sees particles of its own world, and one launch per pass
    covers all worlds.

    Example::

        builder = ModelBuilder()
        SolverSPH.register_custom_attributes(builder)   # optional sph.density/pressure
        builder.add_particle_grid(...)
        model = builder.finalize("cuda:0")
        solver = SolverSPH(model, SolverSPH.Config(smoothing_length=0.02, box_lo=(0,0,0), box_hi=(1,1,1)))
        s0, s1 = model.state(), model.state()
        solver.step(s0, s1, model.control(), None, 1e-4)
    """

    Config = SPHConfig

    def __init__(self, model: Model, config: SPHConfig | list[SPHConfig] | None = None):
        super().__init__(model)
        if model.device.type != "cuda":
            raise RuntimeError("SolverSPH runs on CUDA only (there is no CPU fallback)")
        self._lib = _lib.load()
        self._handle = ctypes.c_void_p()
        self._dt = None
        self.launches_total = 0  # kernels enqueued by this solver's library calls (step, rollout, adjoint)
        if isinstance(config, (list, tuple)):
            self._init_worlds(model, list(config))
            return
        self.world_configs = None
        self.config = config if config is not None else SPHConfig()
        if self.config.smoothing_length <= 0.0:
            raise ValueError("smoothing_length must be positive")
        self.grid_dims = self.config.resolved_grid_dims()
        dims = (ctypes.c_int * 3)(*self.grid_dims)
        _lib.check(
            self._lib.nsph_sph_create(model.device.index or 0, int(model.particle_count), ctypes.byref(dims),
                                      ctypes.byref(self._handle)),
            "SolverSPH()",
        )
        self._params = self.config.params(0.0, model.particle_max_velocity)
        self.set_arithmetic(self.config.arithmetic)

    def set_arithmetic(self, mode: str) -> None:
        """"exact" or "fast" arithmetic of the plain step (see SPHConfig)."""
        modes = {"exact": 0, "fast": 1}
        if mode not in modes:
            raise ValueError(f"arithmetic must be one of {sorted(modes)}, got {mode!r}")
        _lib.check(self._lib.nsph_sph_set_arithmetic(self._handle, modes[mode]), "SolverSPH.set_arithmetic")
        self.arithmetic = mode

    def _init_worlds(self, model: Model, configs: list[SPHConfig]) -> None:
        if len(configs) != model.world_count:
            raise ValueError(f"{len(configs)} configs for {model.world_count} worlds")
        for c in configs:
            if c.smoothing_length <= 0.0:
                raise ValueError("smoothing_length must be positive")
        self.world_configs = configs
        self.config = configs[0]
        self.world_grid_dims = [c.resolved_grid_dims(tight=True) for c in configs]
        self.grid_dims = None
        dims = (ctypes.c_int * (3 * len(configs)))(*[d for wd in self.world_grid_dims for d in wd])
        _lib.check(
            self._lib.nsph_sph_create_worlds(model.device.index or 0, int(model.particle_count), len(configs), dims,
                                             ctypes.byref(self._handle)),
            "SolverSPH()",
        )
        self._upload_world_params()

    def _upload_world_params(self) -> None:
        arr = (_lib.NsphSphParams * len(self.world_configs))()
        for w, c in enumerate(self.world_configs):
            arr[w] = c.params(0.0, self.model.particle_max_velocity)
        _lib.check(self._lib.nsph_sph_set_world_params(self._handle, arr, len(self.world_configs)),
                   "SolverSPH.set_world_params")
        self._params = arr[0]

    @property
    def batched(self) -> bool:
        """True in batched-worlds mode (one config per world)."""
        return self.world_configs is not None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.nsph_sph_destroy(h)
            self._handle = None

    # ------------------------------------------------------------------
    def params_for(self, dt: float) -> _lib.NsphSphParams:
        """The fp32 parameter block of a step with time step dt."""
        if self._dt != dt:
            self._params.dt = float(F32(dt))
            self._dt = dt
        return self._params

    def step(self, state_in: State, state_out: State, control: Control | None, contacts, dt: float) -> None:
        """Advance one WCSPH step from state_in to state_out.

        Args:
            state_in: positions/velocities at time t (and external forces in
                ``particle_f`` when ``config.apply_particle_f``).
            state_out: receives positions/velocities at t + dt; when the model
                registered the ``sph`` state attributes, also the density and
                pressure of the step (``state_out.sph.density`` / ``.pressure``).
                Must not share arrays with state_in.
            control: unused (a particle fluid has no control inputs); None is
                accepted as in the reference.
            contacts: must be None: particle-shape contacts are not part of
                this solver (the box boundary is handled in the kernel).
            dt: time step [s].
        """
        if contacts is not None:
            raise ValueError("SolverSPH does not consume Contacts; pass contacts=None")
        model = self.model
        n = model.particle_count
        if n == 0:
            return
        for name, t in (("state_in.particle_q", state_in.particle_q), ("state_in.particle_qd", state_in.particle_qd),
                        ("state_out.particle_q", state_out.particle_q),
                        ("state_out.particle_qd", state_out.particle_qd)):
            _require_cuda(t, name)
            if t.dtype != torch.float32 or tuple(t.shape) != (n, 3) or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous ({n}, 3) float32 tensor")
        f_ext = state_in.particle_f if (self.config.apply_particle_f and state_in.particle_f is not None) else None
        if torch.is_grad_enabled() and any(t is not None and t.requires_grad
                                           for t in (state_in.particle_q, state_in.particle_qd, f_ext)):
            # differentiable step (models finalized with requires_grad=True):
            # state_out's arrays become the outputs of an autograd node whose
            # backward is the hand-written adjoint, as wp.Tape records a step
            # (newton/solvers.py:359-395). Inactive particles keep state_in's
            # velocity; the sph namespace outputs are not written.
            from .sph_diff import sph_step

            if self.batched:
                raise ValueError("differentiable steps need a single-world solver")
            state_out.particle_q, state_out.particle_qd = sph_step(
                self, state_in.particle_q, state_in.particle_qd, dt, None, f_ext)
            return
        ns = getattr(state_out, "sph", None)
        rho = getattr(ns, "density", None) if ns is not None else None
        prs = getattr(ns, "pressure", None) if ns is not None else None
        acc = getattr(ns, "acceleration", None) if ns is not None else None
        if self.batched:
            st = self._lib.nsph_sph_step_worlds(
                self._handle, float(F32(dt)), n, state_in.particle_q.data_ptr(), state_in.particle_qd.data_ptr(),
                _lib.ptr(f_ext), model.particle_mass.data_ptr(), model.particle_inv_mass.data_ptr(),
                model.particle_flags.data_ptr(), model.particle_world.data_ptr(), model.gravity.data_ptr(),
                int(model.gravity.shape[0]), state_out.particle_q.data_ptr(), state_out.particle_qd.data_ptr(),
                _lib.ptr(rho), _lib.ptr(prs), _lib.ptr(acc), _lib.stream_handle(model.device))
            _lib.check(st, "SolverSPH.step")
            self.launches_total += self.last_launches
            return
        p = self.params_for(dt)
        st = self._lib.nsph_sph_step(
            self._handle,
            ctypes.byref(p),
            n,
            state_in.particle_q.data_ptr(),
            state_in.particle_qd.data_ptr(),
            _lib.ptr(f_ext),
            model.particle_mass.data_ptr(),
            model.particle_inv_mass.data_ptr(),
            model.particle_flags.data_ptr(),
            model.particle_world.data_ptr(),
            model.gravity.data_ptr(),
            int(model.gravity.shape[0]),
            state_out.particle_q.data_ptr(),
            state_out.particle_qd.data_ptr(),
            _lib.ptr(rho),
            _lib.ptr(prs),
            _lib.ptr(acc),
            _lib.stream_handle(model.device),
        )
        _lib.check(st, "SolverSPH.step")
        self.launches_total += self.last_launches

    # ---- adjoint ---------------------------------------------------------
    def enable_adjoint(self) -> None:
        """Allocate the adjoint scratch (36 bytes per particle); called on
        demand by :meth:`step_backward`, outside graph capture."""
        if self.batched:
            raise ValueError("the adjoint supports single-world solvers only")
        if not getattr(self, "_adjoint_ready", False):
            _lib.check(self._lib.nsph_sph_enable_adjoint(self._handle), "SolverSPH.enable_adjoint")
            self._adjoint_ready = True

    def step_params(self, dt: float, eos_b: float | None = None) -> _lib.NsphSphParams:
        """A private copy of the fp32 parameter block for time step dt, with
        the EOS stiffness B replaced by `eos_b` when given."""
        p = _lib.NsphSphParams()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self.params_for(dt)), ctypes.sizeof(p))
        if eos_b is not None:
            p.eos_b = float(F32(eos_b))
        return p

    def _check_vec(self, t: torch.Tensor, name: str) -> None:
        n = self.model.particle_count
        _require_cuda(t, name)
        if t.dtype != torch.float32 or tuple(t.shape) != (n, 3) or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous ({n}, 3) float32 tensor")

    def step_raw(self, x_in: torch.Tensor, v_in: torch.Tensor, x_out: torch.Tensor, v_out: torch.Tensor,
                 params: _lib.NsphSphParams, f_ext: torch.Tensor | None = None) -> None:
        """One step on plain (N, 3) tensors with an explicit parameter block
        and external force (None = none). v_out keeps its contents for
        inactive particles, as in :meth:`step`."""
        model = self.model
        n = model.particle_count
        if self.batched:
            raise ValueError("step_raw needs a single-world solver")
        for t, name in ((x_in, "x_in"), (v_in, "v_in"), (x_out, "x_out"), (v_out, "v_out")):
            self._check_vec(t, name)
        if f_ext is not None:
            self._check_vec(f_ext, "f_ext")
        st = self._lib.nsph_sph_step(
            self._handle, ctypes.byref(params), n, x_in.data_ptr(), v_in.data_ptr(), _lib.ptr(f_ext),
            model.particle_mass.data_ptr(), model.particle_inv_mass.data_ptr(), model.particle_flags.data_ptr(),
            model.particle_world.data_ptr(), model.gravity.data_ptr(), int(model.gravity.shape[0]),
            x_out.data_ptr(), v_out.data_ptr(), None, None, None, _lib.stream_handle(model.device))
        _lib.check(st, "SolverSPH.step_raw")
        self.launches_total += self.last_launches

    def step_backward_raw(self, x_in: torch.Tensor, v_in: torch.Tensor, params: _lib.NsphSphParams,
                          x_out_grad: torch.Tensor, v_out_grad: torch.Tensor, x_in_grad: torch.Tensor,
                          v_in_grad: torch.Tensor, f_ext: torch.Tensor | None = None,
                          rho_out_grad: torch.Tensor | None = None, f_ext_grad: torch.Tensor | None = None,
                          eos_b_grad: torch.Tensor | None = None) -> None:
        """nsph_sph_step_adjoint on plain tensors: writes x_in_grad, v_in_grad
        (which may be x_out_grad, v_out_grad themselves) and adds to
        f_ext_grad (N, 3) and eos_b_grad (one float32) when given."""
        model = self.model
        n = model.particle_count
        self.enable_adjoint()
        for t, name in ((x_in, "x_in"), (v_in, "v_in"), (x_out_grad, "x_out_grad"), (v_out_grad, "v_out_grad"),
                        (x_in_grad, "x_in_grad"), (v_in_grad, "v_in_grad")):
            self._check_vec(t, name)
        for t, name in ((f_ext, "f_ext"), (f_ext_grad, "f_ext_grad")):
            if t is not None:
                self._check_vec(t, name)
        if rho_out_grad is not None and (rho_out_grad.dtype != torch.float32 or tuple(rho_out_grad.shape) != (n,)
                                         or not rho_out_grad.is_cuda or not rho_out_grad.is_contiguous()):
            raise ValueError(f"rho_out_grad must be a contiguous ({n},) float32 CUDA tensor")
        if eos_b_grad is not None and (eos_b_grad.dtype != torch.float32 or eos_b_grad.numel() != 1
                                       or not eos_b_grad.is_cuda):
            raise ValueError("eos_b_grad must be a one-element float32 CUDA tensor")
        st = self._lib.nsph_sph_step_adjoint(
            self._handle, ctypes.byref(params), n, x_in.data_ptr(), v_in.data_ptr(), _lib.ptr(f_ext),
            model.particle_mass.data_ptr(), model.particle_inv_mass.data_ptr(), model.particle_flags.data_ptr(),
            model.particle_world.data_ptr(), model.gravity.data_ptr(), int(model.gravity.shape[0]),
            x_out_grad.data_ptr(), v_out_grad.data_ptr(), _lib.ptr(rho_out_grad), x_in_grad.data_ptr(),
            v_in_grad.data_ptr(), _lib.ptr(f_ext_grad), _lib.ptr(eos_b_grad), _lib.stream_handle(model.device))
        _lib.check(st, "SolverSPH.step_backward")
        self.launches_total += self.last_launches

    def _model_ptrs(self):
        m = self.model
        return (m.particle_mass.data_ptr(), m.particle_inv_mass.data_ptr(), m.particle_flags.data_ptr(),
                m.particle_world.data_ptr(), m.gravity.data_ptr(), int(m.gravity.shape[0]))

    def rollout_raw(self, x0: torch.Tensor, v0: torch.Tensor, x_traj: torch.Tensor, v_traj: torch.Tensor,
                    params: _lib.NsphSphParams, f_ext: torch.Tensor | None = None) -> None:
        """nsph_sph_rollout: x_traj.shape[0] steps from (x0, v0); the state
        after step t goes to x_traj[t], v_traj[t] ((steps, N, 3) float32)."""
        n = self.model.particle_count
        if self.batched:
            raise ValueError("rollout_raw needs a single-world solver")
        for t, name in ((x0, "x0"), (v0, "v0")):
            self._check_vec(t, name)
        steps = int(x_traj.shape[0])
        for t, name in ((x_traj, "x_traj"), (v_traj, "v_traj")):
            _require_cuda(t, name)
            if t.dtype != torch.float32 or tuple(t.shape) != (steps, n, 3) or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous ({steps}, {n}, 3) float32 tensor")
        if f_ext is not None:
            self._check_vec(f_ext, "f_ext")
        st = self._lib.nsph_sph_rollout(self._handle, ctypes.byref(params), n, steps, x0.data_ptr(), v0.data_ptr(),
                                        _lib.ptr(f_ext), *self._model_ptrs(), x_traj.data_ptr(), v_traj.data_ptr(),
                                        _lib.stream_handle(self.model.device))
        _lib.check(st, "SolverSPH.rollout")
        self.launches_total += self.last_launches

    def rollout_backward_raw(self, x_states: torch.Tensor, v_states: torch.Tensor, params: _lib.NsphSphParams,
                             x_grad: torch.Tensor, v_grad: torch.Tensor, f_ext: torch.Tensor | None = None,
                             f_ext_grad: torch.Tensor | None = None, eos_b_grad: torch.Tensor | None = None) -> None:
        """nsph_sph_rollout_adjoint: reverse of x_states.shape[0] steps whose
        input states are x_states[t], v_states[t]; x_grad / v_grad (N, 3) go
        from the last output's gradient to the first input's, in place."""
        n = self.model.particle_count
        self.enable_adjoint()
        steps = int(x_states.shape[0])
        for t, name in ((x_states, "x_states"), (v_states, "v_states")):
            _require_cuda(t, name)
            if t.dtype != torch.float32 or tuple(t.shape) != (steps, n, 3) or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous ({steps}, {n}, 3) float32 tensor")
        for t, name in ((x_grad, "x_grad"), (v_grad, "v_grad")):
            self._check_vec(t, name)
        for t, name in ((f_ext, "f_ext"), (f_ext_grad, "f_ext_grad")):
            if t is not None:
                self._check_vec(t, name)
        if eos_b_grad is not None and (eos_b_grad.dtype != torch.float32 or eos_b_grad.numel() != 1
                                       or not eos_b_grad.is_cuda):
            raise ValueError("eos_b_grad must be a one-element float32 CUDA tensor")
        st = self._lib.nsph_sph_rollout_adjoint(
            self._handle, ctypes.byref(params), n, steps, x_states.data_ptr(), v_states.data_ptr(), _lib.ptr(f_ext),
            *self._model_ptrs(), x_grad.data_ptr(), v_grad.data_ptr(), _lib.ptr(f_ext_grad), _lib.ptr(eos_b_grad),
            _lib.stream_handle(self.model.device))
        _lib.check(st, "SolverSPH.rollout_backward")
        self.launches_total += self.last_launches

    def segment_backward_raw(self, x0: torch.Tensor, v0: torch.Tensor, steps: int, params: _lib.NsphSphParams,
                             x_grad: torch.Tensor, v_grad: torch.Tensor, f_ext: torch.Tensor | None = None,
                             f_ext_grad: torch.Tensor | None = None, eos_b_grad: torch.Tensor | None = None) -> None:
        """nsph_sph_segment_adjoint: recompute `steps` steps from (x0, v0)
        keeping each step's grid and density scratch, then reverse them;
        x_grad / v_grad (N, 3) go from the gradient of the state after
        `steps` steps to that of (x0, v0), in place. Equal, bit for bit, to
        rollout_raw of the segment followed by rollout_backward_raw."""
        n = self.model.particle_count
        self.enable_adjoint()
        for t, name in ((x0, "x0"), (v0, "v0"), (x_grad, "x_grad"), (v_grad, "v_grad")):
            self._check_vec(t, name)
        for t, name in ((f_ext, "f_ext"), (f_ext_grad, "f_ext_grad")):
            if t is not None:
                self._check_vec(t, name)
        if eos_b_grad is not None and (eos_b_grad.dtype != torch.float32 or eos_b_grad.numel() != 1
                                       or not eos_b_grad.is_cuda):
            raise ValueError("eos_b_grad must be a one-element float32 CUDA tensor")
        st = self._lib.nsph_sph_segment_adjoint(
            self._handle, ctypes.byref(params), n, int(steps), x0.data_ptr(), v0.data_ptr(), _lib.ptr(f_ext),
            *self._model_ptrs(), x_grad.data_ptr(), v_grad.data_ptr(), _lib.ptr(f_ext_grad), _lib.ptr(eos_b_grad),
            _lib.stream_handle(self.model.device))
        _lib.check(st, "SolverSPH.segment_backward")
        self.launches_total += self.last_launches

    def reserve_segment(self, steps: int) -> None:
        """Allocate the segment tape of segment_backward_raw for up to
        `steps` steps (outside graph capture)."""
        _lib.check(self._lib.nsph_sph_reserve_segment(self._handle, int(steps)), "SolverSPH.reserve_segment")

    # ---- surrogate ---------------------------------------------------------
    def enable_surrogate(self) -> None:
        """Allocate the surrogate's feature scratch (96 bytes per particle);
        outside graph capture."""
        if self.batched:
            raise ValueError("the surrogate supports single-world solvers only")
        if not getattr(self, "_surrogate_ready", False):
            _lib.check(self._lib.nsph_sph_enable_surrogate(self._handle), "SolverSPH.enable_surrogate")
            self._surrogate_ready = True

    def features_raw(self, x: torch.Tensor, v: torch.Tensor, feat_out: torch.Tensor | None = None,
                     acc_out: torch.Tensor | None = None, rho_out: torch.Tensor | None = None,
                     params: _lib.NsphSphParams | None = None) -> None:
        """nsph_sph_features on (x, v): the 16 surrogate features (N, 16) and
        the SPH acceleration + XSPH sum (N, 6) of each particle."""
        n = self.model.particle_count
        self.enable_surrogate()
        self._check_vec(x, "x")
        self._check_vec(v, "v")
        for t, name, w in ((feat_out, "feat_out", 16), (acc_out, "acc_out", 6)):
            if t is not None and (t.dtype != torch.float32 or tuple(t.shape) != (n, w) or not t.is_contiguous()
                                  or not t.is_cuda):
                raise ValueError(f"{name} must be a contiguous ({n}, {w}) float32 CUDA tensor")
        p = params if params is not None else self.step_params(self._dt or 0.0)
        st = self._lib.nsph_sph_features(self._handle, ctypes.byref(p), n, x.data_ptr(), v.data_ptr(),
                                         *self._model_ptrs(), _lib.ptr(feat_out), _lib.ptr(acc_out), _lib.ptr(rho_out),
                                         _lib.stream_handle(self.model.device))
        _lib.check(st, "SolverSPH.features")
        self.launches_total += self.last_launches

    def step_surrogate_raw(self, x_in: torch.Tensor, v_in: torch.Tensor, x_out: torch.Tensor, v_out: torch.Tensor,
                           params: _lib.NsphSphParams, model, acc_scale: float, stats: torch.Tensor,
                           f_ext: torch.Tensor | None = None, rho_out: torch.Tensor | None = None,
                           p_out: torch.Tensor | None = None) -> None:
        """nsph_sph_step_surrogate: one corrected step of params.dt with the
        MLP `model` (a SurrogateModel); stats: device float[4] monitor."""
        n = self.model.particle_count
        self.enable_surrogate()
        for t, name in ((x_in, "x_in"), (v_in, "v_in"), (x_out, "x_out"), (v_out, "v_out")):
            self._check_vec(t, name)
        if stats.dtype != torch.float32 or stats.numel() < 4 or not stats.is_cuda:
            raise ValueError("stats must be a float32 CUDA tensor of 4 entries")
        st = self._lib.nsph_sph_step_surrogate(
            self._handle, ctypes.byref(params), model.buf.data_ptr(), float(acc_scale), n, x_in.data_ptr(),
            v_in.data_ptr(), _lib.ptr(f_ext), *self._model_ptrs(), x_out.data_ptr(), v_out.data_ptr(),
            _lib.ptr(rho_out), _lib.ptr(p_out), stats.data_ptr(), _lib.stream_handle(self.model.device))
        _lib.check(st, "SolverSPH.step_surrogate")
        self.launches_total += self.last_launches

    def step_backward(self, state_in: State, dt: float, x_out_grad: torch.Tensor, v_out_grad: torch.Tensor,
                      rho_out_grad: torch.Tensor | None = None) -> dict[str, torch.Tensor]:
        """Reverse of ``step(state_in, state_out, None, None, dt)``: the
        gradients of a scalar with respect to the step's inputs, given its
        gradients with respect to state_out's positions, velocities (and
        optionally densities). Replaces ``wp.Tape.backward`` over one step
        (newton/solvers.py:359-395).

        Returns:
            {"particle_q": (N,3), "particle_qd": (N,3), "particle_f": (N,3)
             (only with ``config.apply_particle_f`` and state_in.particle_f),
             "eos_b": (1,)}
        """
        n = self.model.particle_count
        dev = self.model.device
        f_ext = state_in.particle_f if (self.config.apply_particle_f and state_in.particle_f is not None) else None
        xg = torch.empty((n, 3), dtype=torch.float32, device=dev)
        vg = torch.empty_like(xg)
        fg = torch.zeros_like(xg) if f_ext is not None else None
        bg = torch.zeros(1, dtype=torch.float32, device=dev)
        self.step_backward_raw(state_in.particle_q, state_in.particle_qd, self.step_params(dt),
                               x_out_grad.contiguous(), v_out_grad.contiguous(), xg, vg, f_ext=f_ext,
                               rho_out_grad=rho_out_grad, f_ext_grad=fg, eos_b_grad=bg)
        out = {"particle_q": xg, "particle_qd": vg, "eos_b": bg}
        if fg is not None:
            out["particle_f"] = fg
        return out

    def notify_model_changed(self, flags: int) -> None:
        """MODEL_PROPERTIES re-reads particle_max_velocity; gravity needs no
        action (read on the device every step)."""
        if flags & SolverNotifyFlags.MODEL_PROPERTIES:
            if self.batched:
                self._upload_world_params()
            else:
                self._params = self.config.params(0.0 if self._dt is None else self._dt,
                                                  self.model.particle_max_velocity)

    @classmethod
    def register_custom_attributes(cls, builder: ModelBuilder) -> None:
        """Declare the per-particle state outputs ``sph:density`` and
        ``sph:pressure`` (float32), following the solver-namespace pattern of
        SolverImplicitMPM.register_custom_attributes."""
        for name in ("density", "pressure"):
            builder.add_custom_attribute(
                ModelBuilder.CustomAttribute(name, frequency=Model.AttributeFrequency.PARTICLE,
                                             assignment=Model.AttributeAssignment.STATE, dtype=torch.float32,
                                             default=0.0, namespace="sph")
            )

    # ---- inspection of the last step -----------------------------------
    def neighbors(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Neighbour lists of the last step's positions, original order:
        ids[offsets[i]:offsets[i+1]] are the active particles within h of
        particle i (self included), in the grid query order.

        Returns:
            (offsets int64 (N+1,), ids int32)
        """
        n = self.model.particle_count
        dev = self.model.device
        counts = torch.zeros(n, dtype=torch.int32, device=dev)
        stream = _lib.stream_handle(dev)
        p = self._params
        _lib.check(self._lib.nsph_sph_neighbors(self._handle, ctypes.byref(p), counts.data_ptr(), None, None, stream),
                   "SolverSPH.neighbors")
        offsets = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        offsets[1:] = torch.cumsum(counts.to(torch.int64), 0)
        total = int(offsets[-1].item())
        ids = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
        _lib.check(self._lib.nsph_sph_neighbors(self._handle, ctypes.byref(p), None, offsets.data_ptr(),
                                                ids.data_ptr(), stream), "SolverSPH.neighbors")
        return offsets, ids[:total]

    def grid_arrays(self) -> dict[str, torch.Tensor]:
        """Copies of the last step's grid: sorted cell ids, sorted point ids
        (the permutation), cell_starts and cell_ends."""
        from ..hashgrid import _view_int

        v = _lib.NsphGridView()
        _lib.check(self._lib.nsph_sph_get_grid_view(self._handle, ctypes.byref(v)), "SolverSPH.grid_arrays")
        dev = self.model.device
        if self.batched:  # cell tables of all worlds are one large table: return the sort only
            return {
                "point_cells": _view_int(v.point_cells, v.num_points, dev).clone(),
                "point_ids": _view_int(v.point_ids, v.num_points, dev).clone(),
            }
        nc = v.dim_x * v.dim_y * v.dim_z
        return {
            "point_cells": _view_int(v.point_cells, v.num_points, dev).clone(),
            "point_ids": _view_int(v.point_ids, v.num_points, dev).clone(),
            "cell_starts": _view_int(v.cell_starts, nc, dev, v.cell_stride).clone(),
            "cell_ends": _view_int(v.cell_ends, nc, dev, v.cell_stride).clone(),
        }

    def enable_phase_timing(self, enable: bool = True) -> None:
        """Record CUDA events around the build, density and force phases of
        every later step (also inside captured CUDA graphs). Call outside a
        capture."""
        _lib.check(self._lib.nsph_sph_enable_phase_timing(self._handle, int(bool(enable))),
                   "SolverSPH.enable_phase_timing")

    def phase_times(self) -> tuple[float, float, float]:
        """(build, density, force) milliseconds of the last executed step;
        waits for that step to finish."""
        ms = (ctypes.c_float * 3)()
        _lib.check(self._lib.nsph_sph_phase_times(self._handle, ctypes.byref(ms)), "SolverSPH.phase_times")
        return float(ms[0]), float(ms[1]), float(ms[2])

    def adjoint_phase_times(self) -> tuple[float, float, float, float, float]:
        """(build, density, force recompute + integrate reverse, pair gather,
        density gather) milliseconds of the last executed adjoint step; waits
        for it. Needs :meth:`enable_phase_timing`. A step reversed by
        :meth:`segment_backward_raw` reads its build and density from the
        segment tape, so those two phases are 0 there."""
        ms = (ctypes.c_float * 5)()
        _lib.check(self._lib.nsph_sph_adjoint_phase_times(self._handle, ctypes.byref(ms)),
                   "SolverSPH.adjoint_phase_times")
        return tuple(float(v) for v in ms)

    def set_surrogate_wait_limit(self, polls: int = -1) -> None:
        """Polls of each tensor-core completion wait of the surrogate step (-1:
        the library default). 0 makes the waits give up at once, which
        exercises the timeout path (uncorrected integration, status bit)."""
        self.enable_surrogate()
        _lib.check(self._lib.nsph_sph_set_surrogate_wait_limit(self._handle, int(polls)),
                   "SolverSPH.set_surrogate_wait_limit")

    def set_surrogate_launch(self, ctas_per_sm: int = 0, tiles_per_cta: int = 0) -> None:
        """Launch shape of the surrogate step's fused kernel: resident CTAs
        per SM and 128-particle tiles per CTA (1 or 2; 0: the defaults). See
        nsph_sph_set_surrogate_launch; results do not change."""
        self.enable_surrogate()
        _lib.check(self._lib.nsph_sph_set_surrogate_launch(self._handle, int(ctas_per_sm), int(tiles_per_cta)),
                   "SolverSPH.set_surrogate_launch")

    def surrogate_phase_times(self) -> tuple[float, float, float, float]:
        """(build, density, fused features + MLP + integrate, compression
        reduction) milliseconds of the last executed surrogate step; waits for
        it. Needs :meth:`enable_phase_timing`."""
        ms = (ctypes.c_float * 4)()
        _lib.check(self._lib.nsph_sph_surrogate_phase_times(self._handle, ctypes.byref(ms)),
                   "SolverSPH.surrogate_phase_times")
        return tuple(float(v) for v in ms)

    def set_launch(self, threads: int = 0, blocks_per_sm: int = -1) -> None:
        """Launch shape of the density and force passes (see nsph_sph_set_launch)."""
        _lib.check(self._lib.nsph_sph_set_launch(self._handle, int(threads), int(blocks_per_sm)),
                   "SolverSPH.set_launch")
        self.launch = (int(threads), int(blocks_per_sm))

    def autotune(self, state_in: State, state_out: State, dt: float, candidates=None, repeats: int = 3) -> dict:
        """Pick the fastest launch shape of the neighbour passes.

        Runs `repeats` steps state_in -> state_out per candidate (threads per
        block, persistent blocks per SM; 0 = one thread per particle), timed
        on the device with the library's phase events, and keeps the fastest
        density + force time. Outside a CUDA graph capture only. Results do not
        depend on the launch shape.

        Returns:
            {(threads, blocks_per_sm): ms of density + force per step, ...,
             "best": (threads, blocks_per_sm)}
        """
        if candidates is None:
            candidates = [(t, b) for t in (128, 256) for b in (0, 2, 3, 4, 8)]
        self.enable_phase_timing(True)
        results = {}
        for t, b in candidates:
            self.set_launch(t, b)
            self.step(state_in, state_out, None, None, dt)  # warm-up of this shape
            best = float("inf")
            for _ in range(repeats):
                self.step(state_in, state_out, None, None, dt)
                _, d, f = self.phase_times()
                best = min(best, d + f)
            results[(t, b)] = best
        choice = min(results, key=results.get)
        self.set_launch(*choice)
        results["best"] = choice
        return results

    @property
    def last_launches(self) -> int:
        """Kernels launched by the last step."""
        return int(self._lib.nsph_sph_last_launches(self._handle))

    def status(self) -> int:
        """Device status word (NSPH_STATUS_* bits) accumulated since the last
        reset; synchronises the current stream."""
        s = ctypes.c_uint(0)
        _lib.check(self._lib.nsph_sph_status(self._handle, ctypes.byref(s), _lib.stream_handle(self.model.device)),
                   "SolverSPH.status")
        return int(s.value)

    def reset_status(self) -> None:
        _lib.check(self._lib.nsph_sph_reset_status(self._handle, _lib.stream_handle(self.model.device)),
                   "SolverSPH.reset_status")


__all__ = ["SPHConfig", "SolverSPH"]
