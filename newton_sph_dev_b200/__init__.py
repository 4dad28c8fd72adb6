"""newton_sph_dev_b200 — Newton's particle-fluid hot path on B200 (sm_100a).

Drop-in for the particle part of NVIDIA Newton's API:

- ``ModelBuilder`` / ``Model`` / ``State`` / ``Control`` (torch tensors),
- ``HashGrid`` (the ``wp.HashGrid`` build/query semantics),
- ``solvers.SolverBase`` (``integrate_particles``) and ``solvers.SolverSPH``
  (weakly-compressible SPH: hash-grid neighbour search, density/EOS,
  pressure + XSPH forces, integration),
- ``solvers.SolverXPBD`` / ``solvers.SolverSemiImplicit`` (their particle
  paths: particle-particle contacts on the grid, particle contacts with
  static planes, spheres, boxes, capsules, cylinders, cones and ellipsoids
  through ``Model.collide``),
- ``sensors.SensorRaycast`` (the depth camera's particle raycast on the grid),
- ``recording`` (state dumps to resume from, trajectory recording, JSONL
  metrics).

All compute runs in libnsph.so (hand-written CUDA for sm_100a, C ABI in
include/nsph.h); there is no CPU fallback.
"""

from . import recording, sensors, solvers
from .geometry import GeoType, ParticleFlags, ShapeFlags
from .hashgrid import HashGrid
from .sim import Contacts, Control, Model, ModelBuilder, State

__version__ = "0.1.0"

__all__ = ["Contacts", "Control", "GeoType", "HashGrid", "Model", "ModelBuilder", "ParticleFlags", "ShapeFlags", "State",
           "recording", "sensors", "solvers"]
