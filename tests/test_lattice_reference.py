"""ModelBuilder.add_particle_grid against the reference's own method.

tests/golden/lattice_reference.npz holds what the reference's
add_particle_grid (newton/_src/sim/builder.py:8037-8137), compiled from its
source by tests/golden/make_lattice_golden.py, passes to add_particles for
four grids: offsets, a 90-degree and a general rotation, jitter, radius
draws with radius_std > 0, flags, and particles already in the builder
(the seed rule default_rng(42 + count)). This library's builder must give
the same positions, velocities, radii, masses and flags bit for bit, before
and after the float32 conversion of finalize.
"""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "lattice_reference.npz"

_spec = importlib.util.spec_from_file_location("make_lattice_golden", GOLDEN.parent / "make_lattice_golden.py")
_mod = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mod)
CASES = _mod.CASES


@pytest.mark.parametrize("case", range(len(CASES)))
def test_builder_matches_reference_method(case):
    import newton_sph_dev_b200 as nsph

    d = np.load(GOLDEN)
    kw, existing = CASES[case]
    b = nsph.ModelBuilder()
    if existing:
        b.add_particles(pos=np.zeros((existing, 3)), vel=np.zeros((existing, 3)), mass=np.ones(existing))
    b.add_particle_grid(**kw)
    n = d[f"case{case}_points"].shape[0]
    np.testing.assert_array_equal(b.particle_q[existing:], d[f"case{case}_points"])
    np.testing.assert_array_equal(b.particle_qd[existing:], d[f"case{case}_vel"])
    np.testing.assert_array_equal(b.particle_radius[existing:], d[f"case{case}_radius"])
    np.testing.assert_array_equal(b.particle_mass[existing:], d[f"case{case}_mass"])
    flags = d[f"case{case}_flags"]
    want_flags = flags if flags.size else np.full(n, int(nsph.ParticleFlags.ACTIVE))
    np.testing.assert_array_equal(b.particle_flags[existing:], want_flags)
    m = b.finalize("cpu")
    np.testing.assert_array_equal(m.particle_q.numpy()[existing:], d[f"case{case}_points"].astype(np.float32))
    np.testing.assert_array_equal(m.particle_radius.numpy()[existing:], d[f"case{case}_radius"].astype(np.float32))


def test_fixture_is_current_when_the_reference_is_present():
    """Where the reference tree exists, regenerating the fixture gives the
    committed one (the method and the generator have not drifted)."""
    if not _mod.REFERENCE_BUILDER.exists():
        pytest.skip("reference tree not present")
    fn, lo, hi = _mod.reference_add_particle_grid()
    d = np.load(GOLDEN)
    assert [lo, hi] == d["source_lines"].tolist()
    for i, (kw, existing) in enumerate(CASES):
        rec = _mod._Recorder(existing)
        fn(rec, **kw)
        np.testing.assert_array_equal(np.asarray(rec.calls[0]["pos"]), d[f"case{i}_points"])
        np.testing.assert_array_equal(np.asarray(rec.calls[0]["radius"]), d[f"case{i}_radius"])
