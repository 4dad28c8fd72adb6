"""Batched worlds on the GPU: several independent scenes (Newton worlds,
newton/_src/sim/builder.py:2815-2909) in one SolverSPH with one config per
world. Every world must give exactly what the oracle gives for that world run
alone (its own grid and parameters): sort permutation, neighbour lists and
the fp32 step, bit for bit. The worlds overlap in space, so any leak between
worlds would change the results.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"

SPECS = [  # (lattice shape, spacing, velocity std)
    ((8, 8, 8), 0.010, 0.05),
    ((6, 7, 5), 0.008, 0.10),
    ((10, 4, 6), 0.012, 0.0),
    ((5, 5, 5), 0.006, 0.20),
    ((3, 3, 3), 0.010, 0.0),
]


def worlds_scene(specs, device, box=0.2, seed=0):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    b = nsph.ModelBuilder()
    SolverSPH.register_custom_attributes(b)
    b.add_custom_attribute(nsph.ModelBuilder.CustomAttribute(
        "acceleration", frequency=nsph.Model.AttributeFrequency.PARTICLE,
        assignment=nsph.Model.AttributeAssignment.STATE, dtype=torch.float32, namespace="sph", width=3))
    cfgs = []
    for shape, s, _ in specs:
        b.begin_world()
        b.add_particle_grid(pos=(s / 2, s / 2, s / 2), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=shape[0],
                            dim_y=shape[1], dim_z=shape[2], cell_x=s, cell_y=s, cell_z=s, mass=1000.0 * s**3,
                            jitter=0.2 * s)
        b.end_world()
        cfgs.append(SolverSPH.Config(smoothing_length=2 * s, box_lo=(0.0, 0.0, 0.0), box_hi=(box, box, box)))
    model = b.finalize(device)
    rng = np.random.default_rng(seed)
    world = model.particle_world.cpu().numpy()
    v = np.zeros((model.particle_count, 3), np.float32)
    for w, (_, _, vs) in enumerate(specs):
        sel = world == w
        v[sel] = rng.normal(0, vs, (int(sel.sum()), 3)) if vs > 0 else 0.0
    model.particle_qd.copy_(torch.from_numpy(v))
    return model, cfgs


def test_worlds_match_oracle_per_world(oracle_mod):
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfgs = worlds_scene(SPECS, DEV)
    n = model.particle_count
    rng = np.random.default_rng(4)
    flags = np.ones(n, np.int32)
    flags[rng.choice(n, 15, replace=False)] = 0
    mass = model.particle_mass.cpu().numpy()
    mass[rng.choice(n, 10, replace=False)] = 0.0
    inv = np.divide(1.0, mass, out=np.zeros_like(mass), where=mass != 0).astype(np.float32)
    model.particle_flags.copy_(torch.from_numpy(flags))
    model.particle_mass.copy_(torch.from_numpy(mass))
    model.particle_inv_mass.copy_(torch.from_numpy(inv))
    model.set_gravity(np.array([[0, 0, -9.81], [0, -3.0, 0], [1.0, 0, -9.81], [0, 0, 0], [0, 0, 9.81]], np.float32))

    solver = SolverSPH(model, cfgs)
    assert solver.batched
    dt = 1e-4
    s0, s1 = model.state(), model.state()
    s0.particle_f.normal_(0, 1e-4)
    s1.particle_qd.fill_(-3.0)
    v_init = s1.particle_qd.cpu().numpy()
    solver.step(s0, s1, None, None, dt)
    torch.cuda.synchronize()

    x = s0.particle_q.cpu().numpy()
    v = s0.particle_qd.cpu().numpy()
    f = s0.particle_f.cpu().numpy()
    world = model.particle_world.cpu().numpy()
    grav = model.gravity.cpu().numpy()
    got = {"x": s1.particle_q.cpu().numpy(), "v": s1.particle_qd.cpu().numpy(),
           "rho": s1.sph.density.cpu().numpy(), "p": s1.sph.pressure.cpu().numpy(),
           "a": s1.sph.acceleration.cpu().numpy()}
    off, ids = solver.neighbors()
    off, ids = off.cpu().numpy(), ids.cpu().numpy()
    perm = solver.grid_arrays()["point_ids"].cpu().numpy()
    expect_perm = []
    for w, cfg in enumerate(cfgs):
        sel = np.nonzero(world == w)[0]
        consts = cfg.constants(dt, model.particle_max_velocity)
        dims = cfg.resolved_grid_dims(tight=True)
        r = oracle_mod.sph_step(consts, dims, x[sel], v[sel], mass[sel], inv[sel], flags[sel],
                                np.zeros(len(sel), np.int32), grav[w:w + 1], f_ext=f[sel], v_out_init=v_init[sel],
                                precision="f32")
        for k in got:
            np.testing.assert_array_equal(got[k][sel], r[k], err_msg=f"world {w} {k}")
        roff, rids = oracle_mod.sph_neighbors(consts["f32"], dims, x[sel], flags[sel])
        for li, gi in enumerate(sel):
            np.testing.assert_array_equal(ids[off[gi]:off[gi + 1]], sel[rids[roff[li]:roff[li + 1]]],
                                          err_msg=f"world {w} particle {gi}")
        g = oracle_mod.grid_build(x[sel], float(consts["f32"]["cell_width"]), dims)
        expect_perm.append(sel[g["point_ids"]])
    np.testing.assert_array_equal(perm, np.concatenate(expect_perm))


def test_worlds_graph_replay_and_config_checks():
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfgs = worlds_scene(SPECS[:3], DEV)
    with pytest.raises(ValueError):
        SolverSPH(model, cfgs[:2])
    solver = SolverSPH(model, cfgs)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, 1e-4)
    ref0, ref1 = model.state(), model.state()
    ref0.assign(s0)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        solver.step(s0, s1, None, None, 1e-4)
    graph.replay()
    solver.step(ref0, ref1, None, None, 1e-4)
    torch.cuda.synchronize()
    assert torch.equal(s1.particle_q, ref1.particle_q) and torch.equal(s1.particle_qd, ref1.particle_qd)
    assert solver.status() == 0
