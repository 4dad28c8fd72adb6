"""Generate tests/golden/lattice_reference.npz by running the reference's own
ModelBuilder.add_particle_grid (newton/_src/sim/builder.py:8037-8137).

`import newton` needs warp-lang, which is absent here, so this script takes
the method's source from the reference tree with `ast`, compiles it
unchanged, and calls it on a stand-in `self` that records what the method
passes to `add_particles`. `wp.quat_to_matrix` is the one Warp call in the
method; it is supplied by this library's `quat_to_matrix` (the rotation
matrix in fp32), so the fixture pins everything else the method does: the
lattice order, the transform, the seed rule `default_rng(42 + count)`, the
jitter stream and the radius draws.

Run (in a checkout where the reference tree is at /root/reference):
    python tests/golden/make_lattice_golden.py
"""

from __future__ import annotations

import __future__
import ast
import sys
from collections.abc import Sequence
from pathlib import Path
from typing import Any

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

REFERENCE_BUILDER = Path("/root/reference/newton/_src/sim/builder.py")

# (kwargs of add_particle_grid, particles already in the builder)
CASES = [
    (dict(pos=(0.1, -0.2, 0.3), rot=(0.0, 0.0, 0.0, 1.0), vel=(1.0, 2.0, 3.0), dim_x=5, dim_y=4, dim_z=3,
          cell_x=0.01, cell_y=0.02, cell_z=0.03, mass=0.5, jitter=0.004), 0),
    (dict(pos=(-1.0, 0.5, 2.0), rot=(0.0, 0.0, 0.70710677, 0.70710677), vel=(0.0, 0.0, -1.0), dim_x=6, dim_y=3,
          dim_z=4, cell_x=0.05, cell_y=0.05, cell_z=0.05, mass=1.0, jitter=0.01, radius_mean=0.02,
          radius_std=0.003, flags=1), 7),
    (dict(pos=(0.0, 0.0, 0.0), rot=(0.10482848, 0.20965697, 0.31448545, 0.91986218), vel=(0.0, 0.0, 0.0), dim_x=4,
          dim_y=5, dim_z=6, cell_x=0.1, cell_y=0.2, cell_z=0.3, mass=2.0, jitter=0.0), 130),
    (dict(pos=(0.0025, 0.0025, 0.0025), rot=(0.0, 0.0, 0.0, 1.0), vel=(0.0, 0.0, 0.0), dim_x=16, dim_y=16, dim_z=8,
          cell_x=0.005, cell_y=0.005, cell_z=0.005, mass=0.125, jitter=0.001), 0),
]


def reference_add_particle_grid():
    """The reference's add_particle_grid, compiled from its source."""
    tree = ast.parse(REFERENCE_BUILDER.read_text())
    fn = None
    for node in ast.walk(tree):
        if isinstance(node, ast.ClassDef) and node.name == "ModelBuilder":
            for item in node.body:
                if isinstance(item, ast.FunctionDef) and item.name == "add_particle_grid":
                    fn = item
    if fn is None:
        raise RuntimeError("ModelBuilder.add_particle_grid not found in the reference builder")
    fn.decorator_list = []
    mod = ast.Module(body=[fn], type_ignores=[])
    code = compile(mod, str(REFERENCE_BUILDER), "exec", flags=__future__.annotations.compiler_flag,
                   dont_inherit=True)
    from newton_sph_dev_b200.sim.builder import quat_to_matrix

    class _Warp:
        @staticmethod
        def quat_to_matrix(q):
            return quat_to_matrix(q)

    ns = {"np": np, "wp": _Warp(), "Sequence": Sequence, "Any": Any}
    exec(code, ns)
    return ns["add_particle_grid"], fn.lineno, fn.end_lineno


class _Recorder:
    """Stand-in `self`: the builder state the method reads, and a record of
    the add_particles call it makes."""

    def __init__(self, existing: int):
        self.particle_q = [(0.0, 0.0, 0.0)] * existing
        self.default_particle_radius = 0.1
        self.calls = []

    def add_particles(self, pos, vel, mass, radius, flags=None, custom_attributes=None):
        self.calls.append(dict(pos=pos, vel=vel, mass=mass, radius=radius, flags=flags))


def main():
    fn, lo, hi = reference_add_particle_grid()
    out = {}
    for i, (kw, existing) in enumerate(CASES):
        rec = _Recorder(existing)
        fn(rec, **kw)
        (call,) = rec.calls
        n = len(call["pos"])
        out[f"case{i}_points"] = np.asarray(call["pos"], dtype=np.float64).reshape(n, 3)
        out[f"case{i}_vel"] = np.asarray(call["vel"], dtype=np.float64).reshape(n, 3)
        out[f"case{i}_radius"] = np.asarray(call["radius"], dtype=np.float64)
        out[f"case{i}_mass"] = np.asarray(call["mass"], dtype=np.float64)
        fl = call["flags"]
        out[f"case{i}_flags"] = np.asarray(fl if fl is not None else [], dtype=np.int64)
    out["source_lines"] = np.asarray([lo, hi])
    np.savez_compressed(HERE / "lattice_reference.npz", **out)
    print(f"wrote {HERE / 'lattice_reference.npz'} from builder.py:{lo}-{hi}, {len(CASES)} cases")


if __name__ == "__main__":
    main()
