"""Time-varying particle state, mirroring newton/_src/sim/state.py:47-266.

Arrays are torch tensors: ``particle_q`` / ``particle_qd`` / ``particle_f`` of
shape ``(particle_count, 3)`` float32 (the reference's ``wp.array[vec3]``).
"""

from __future__ import annotations

import torch


class AttributeNamespace:
    """Container for namespaced custom attributes (e.g. ``state.sph.density``),
    like Model.AttributeNamespace in newton/_src/sim/model.py."""

    def __init__(self, name: str):
        self._name = name

    def __repr__(self) -> str:
        keys = [k for k in self.__dict__ if not k.startswith("_")]
        return f"AttributeNamespace({self._name!r}, {keys})"


def _copy_tensors(dst, src, prefix: str = "") -> None:
    """Copy every tensor attribute of src into dst (state.py:18-42)."""
    names = {k for k in vars(dst) if not k.startswith("_")} | {k for k in vars(src) if not k.startswith("_")}
    for attr in sorted(names):
        val_dst = getattr(dst, attr, None)
        val_src = getattr(src, attr, None)
        t_dst = isinstance(val_dst, torch.Tensor)
        t_src = isinstance(val_src, torch.Tensor)
        if not t_dst and not t_src:
            continue
        qualified = f"{prefix}{attr}"
        if not t_dst:
            raise ValueError(f"State is missing array for '{qualified}' which is present in the other state.")
        if not t_src:
            raise ValueError(f"Other state is missing array for '{qualified}' which is present in this state.")
        val_dst.copy_(val_src)


class State:
    """Particle positions, velocities and forces of one time level.

    Create states with :meth:`Model.state` rather than directly.
    """

    def __init__(self) -> None:
        self.particle_q: torch.Tensor | None = None
        """Particle positions [m], shape (particle_count, 3), float32."""
        self.particle_qd: torch.Tensor | None = None
        """Particle velocities [m/s], shape (particle_count, 3), float32."""
        self.particle_f: torch.Tensor | None = None
        """Particle forces [N], shape (particle_count, 3), float32 (external
        forces accumulated before the step, cleared by clear_forces)."""

    def clear_forces(self) -> None:
        """Zero ``particle_f`` (state.py:156-167). Not recorded by autograd
        (the forces are inputs, as Warp's tape treats the cleared array)."""
        if self.particle_count:
            with torch.no_grad():
                self.particle_f.zero_()

    def assign(self, other: State) -> None:
        """Copy the arrays of another state into this one (state.py:169-229).

        Used to make an odd number of substeps graph-capturable.

        Raises:
            ValueError: one state has an array (or a namespace holding arrays)
                that the other lacks.
        """
        _copy_tensors(self, other)
        ns_self = {k: v for k, v in vars(self).items() if isinstance(v, AttributeNamespace)}
        ns_other = {k: v for k, v in vars(other).items() if isinstance(v, AttributeNamespace)}
        for name in sorted(ns_self.keys() | ns_other.keys()):
            dst = ns_self.get(name)
            src = ns_other.get(name)
            if dst is None:
                if any(isinstance(v, torch.Tensor) for v in vars(src).values()):
                    raise ValueError(f"State is missing namespace '{name}' which contains arrays in the other state.")
                continue
            if src is None:
                if any(isinstance(v, torch.Tensor) for v in vars(dst).values()):
                    raise ValueError(f"Other state is missing namespace '{name}' which contains arrays in this state.")
                continue
            _copy_tensors(dst, src, prefix=f"{name}.")

    @property
    def requires_grad(self) -> bool:
        """Whether the particle arrays track gradients."""
        if self.particle_q is not None:
            return bool(self.particle_q.requires_grad)
        return False

    @property
    def particle_count(self) -> int:
        """Number of particles in the state."""
        return 0 if self.particle_q is None else int(self.particle_q.shape[0])

    @property
    def body_count(self) -> int:
        return 0


__all__ = ["AttributeNamespace", "State"]
