"""Shared test setup: the `gpu` marker, import paths and common scenes."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(autouse=True)
def _no_bounds_violations(request):
    """With the bounds-checked build loaded (NSPH_LIBRARY=.../libnsph_bounds.so),
    every GPU test must end with no index violation counted by the kernels."""
    import os

    yield
    if not os.environ.get("NSPH_LIBRARY") or request.node.get_closest_marker("gpu") is None:
        return
    from newton_sph_dev_b200 import _lib

    if _lib.bounds_checked():
        import torch

        torch.cuda.synchronize()
        assert _lib.bounds_violations() == 0, "the bounds-checked build counted index violations"


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.build()
    return oracle


def lattice_scene(n_side=(8, 8, 8), spacing=0.01, jitter_frac=0.2, vel_std=0.0, seed=2, origin=None,
                  box_hi=None, device="cpu", register=True):
    """Jittered lattice block (the benchmark scenes' generator) and its SPH config."""
    import torch

    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    s = spacing
    b = nsph.ModelBuilder()
    if register:
        SolverSPH.register_custom_attributes(b)
        b.add_custom_attribute(nsph.ModelBuilder.CustomAttribute(
            "acceleration", frequency=nsph.Model.AttributeFrequency.PARTICLE,
            assignment=nsph.Model.AttributeAssignment.STATE, dtype=torch.float32, default=0.0, namespace="sph",
            width=3))
    origin = origin if origin is not None else (s / 2, s / 2, s / 2)
    b.add_particle_grid(pos=origin, rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=n_side[0], dim_y=n_side[1],
                        dim_z=n_side[2], cell_x=s, cell_y=s, cell_z=s, mass=1000.0 * s**3, jitter=jitter_frac * s)
    model = b.finalize(device)
    if vel_std > 0:
        rng = np.random.default_rng(seed)
        model.particle_qd.copy_(torch.from_numpy(rng.normal(0, vel_std, (model.particle_count, 3)).astype(np.float32)))
    if box_hi is None:
        box_hi = tuple(float(origin[a] + n_side[a] * s + s) for a in range(3))
    cfg = SolverSPH.Config(smoothing_length=2 * s, box_lo=(0.0, 0.0, 0.0), box_hi=box_hi)
    return model, cfg
