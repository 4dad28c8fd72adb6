"""Golden fixtures (tests/golden/sph_small.npz, made by make_golden.py):
the oracle must keep reproducing them (CPU), and the device must match them
(GPU): grid and neighbours bit-exact, the fp32 step bit-exact, the fp64
step within the fp32 tolerances."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

import make_golden  # noqa: E402

GOLD = HERE / "golden" / "sph_small.npz"


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _case(g):
    return {k[3:]: v for k, v in g.items() if k.startswith("in_")}


def test_inputs_regenerate_identically(gold):
    case, _ = make_golden.make_case()
    for k, v in case.items():
        np.testing.assert_array_equal(v, gold[f"in_{k}"], err_msg=k)


def test_oracle_reproduces_golden(oracle_mod, gold):
    case, cfg = make_golden.make_case()
    ans = make_golden.answers(case, cfg, float(gold["dt"]))
    for k, v in ans.items():
        if k.startswith("f64_"):
            np.testing.assert_allclose(v, gold[k], rtol=1e-12, atol=1e-15, err_msg=k)
        else:
            np.testing.assert_array_equal(v, gold[k], err_msg=k)


@pytest.mark.gpu
def test_device_matches_golden(gold):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    case, cfg = make_golden.make_case()
    dev = "cuda:0"
    b = nsph.ModelBuilder()
    SolverSPH.register_custom_attributes(b)
    b.add_custom_attribute(nsph.ModelBuilder.CustomAttribute(
        "acceleration", frequency=nsph.Model.AttributeFrequency.PARTICLE,
        assignment=nsph.Model.AttributeAssignment.STATE, dtype=torch.float32, namespace="sph", width=3))
    b.add_particles(pos=case["x"], vel=case["v"], mass=case["mass"], flags=case["flags"])
    model = b.finalize(dev)
    model.particle_inv_mass.copy_(torch.from_numpy(case["inv_mass"]))
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    s0.particle_f.copy_(torch.from_numpy(case["f_ext"]))
    s1.particle_qd.fill_(-3.0)
    solver.step(s0, s1, None, None, float(gold["dt"]))
    torch.cuda.synchronize()
    assert tuple(solver.grid_dims) == tuple(gold["grid_dims"].tolist())
    g = solver.grid_arrays()
    for k in ("point_cells", "point_ids", "cell_starts", "cell_ends"):
        np.testing.assert_array_equal(g[k].cpu().numpy(), gold[f"grid_{k}"], err_msg=k)
    off, ids = solver.neighbors()
    np.testing.assert_array_equal(off.cpu().numpy(), gold["nbr_offsets"])
    np.testing.assert_array_equal(ids.cpu().numpy(), gold["nbr_ids"])
    got = {"x": s1.particle_q, "v": s1.particle_qd, "rho": s1.sph.density, "p": s1.sph.pressure,
           "a": s1.sph.acceleration}
    for k, t in got.items():
        np.testing.assert_array_equal(t.cpu().numpy(), gold[f"f32_{k}"], err_msg=k)
    rho64 = gold["f64_rho"]
    act = rho64 > 0
    assert np.max(np.abs(got["rho"].cpu().numpy()[act] - rho64[act]) / rho64[act]) < 1e-5
    assert np.max(np.abs(got["x"].cpu().numpy() - gold["f64_x"])) < 1e-6
