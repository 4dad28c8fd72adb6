"""WCSPH step parity on the GPU, through SolverSPH.step -> nsph_sph_step.

Bars:
  - grid cell ids, sort permutation, cell ranges and neighbour lists:
    bit-exact against the CPU oracle;
  - densities, pressures, accelerations, positions and velocities: equal to
    the fp32 oracle (same per-pair arithmetic and summation order), asserted
    bit-exact, and within tolerance of the fp64 oracle: density 1e-5
    relative, positions 1e-5 relative per step and 1e-3 after 100 steps
    (relative to the domain size);
  - Newton's behavioural contracts: free fall, runtime gravity
    (newton/tests/test_runtime_gravity.py:18-67) and runtime gravity under
    CUDA-graph replay (:141-210).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import lattice_scene

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _host(model, state):
    return dict(
        x=state.particle_q.cpu().numpy(),
        v=state.particle_qd.cpu().numpy(),
        f=state.particle_f.cpu().numpy(),
        mass=model.particle_mass.cpu().numpy(),
        inv_mass=model.particle_inv_mass.cpu().numpy(),
        flags=model.particle_flags.cpu().numpy(),
        world=model.particle_world.cpu().numpy(),
        gravity=model.gravity.cpu().numpy(),
    )


def _oracle_step(O, solver, model, h, dt, v_out_init, precision):
    consts = solver.config.constants(dt, model.particle_max_velocity)
    return O.sph_step(consts, solver.grid_dims, h["x"], h["v"], h["mass"], h["inv_mass"], h["flags"], h["world"],
                      h["gravity"], f_ext=h["f"], v_out_init=v_out_init, precision=precision)


def _one_step(model, cfg, dt=1e-4):
    from newton_sph_dev_b200.solvers import SolverSPH

    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    v_init = s1.particle_qd.cpu().numpy()
    solver.step(s0, s1, model.control(), None, dt)
    torch.cuda.synchronize()
    return solver, s0, s1, v_init


@pytest.mark.parametrize("shape,vel", [((12, 12, 12), 0.05), ((32, 32, 32), 0.0), ((20, 7, 13), 0.3)])
def test_step_parity(oracle_mod, shape, vel):
    model, cfg = lattice_scene(shape, vel_std=vel, device=DEV)
    dt = 1e-4
    solver, s0, s1, v_init = _one_step(model, cfg, dt)
    h = _host(model, s0)
    consts = cfg.constants(dt, model.particle_max_velocity)
    # grid and neighbours: bit-exact
    g = solver.grid_arrays()
    ref = oracle_mod.grid_build(h["x"], float(consts["f32"]["cell_width"]), solver.grid_dims)
    for k in ref:
        np.testing.assert_array_equal(g[k].cpu().numpy(), ref[k], err_msg=k)
    off, ids = solver.neighbors()
    roff, rids = oracle_mod.sph_neighbors(consts["f32"], solver.grid_dims, h["x"], h["flags"])
    np.testing.assert_array_equal(off.cpu().numpy(), roff)
    np.testing.assert_array_equal(ids.cpu().numpy(), rids)
    # fp32 oracle: same arithmetic and order -> identical results
    r32 = _oracle_step(oracle_mod, solver, model, h, dt, v_init, "f32")
    np.testing.assert_array_equal(s1.sph.density.cpu().numpy(), r32["rho"])
    np.testing.assert_array_equal(s1.sph.pressure.cpu().numpy(), r32["p"])
    np.testing.assert_array_equal(s1.sph.acceleration.cpu().numpy(), r32["a"])
    np.testing.assert_array_equal(s1.particle_q.cpu().numpy(), r32["x"])
    np.testing.assert_array_equal(s1.particle_qd.cpu().numpy(), r32["v"])
    # fp64 oracle: within tolerance
    r64 = _oracle_step(oracle_mod, solver, model, h, dt, v_init, "f64")
    rho = s1.sph.density.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(rho - r64["rho"]) / r64["rho"]) < 1e-5
    x = s1.particle_q.cpu().numpy().astype(np.float64)
    span = float(np.max(np.abs(r64["x"])))
    assert np.max(np.abs(x - r64["x"])) < 1e-5 * span
    a = s1.sph.acceleration.cpu().numpy().astype(np.float64)
    err = np.linalg.norm(a - r64["a"], axis=1) / np.maximum(r64["a_scale"], 1e-30)
    assert np.median(err) < 1e-5 and np.max(err) < 1e-3  # EOS-conditioned, see test_oracle


def test_inactive_and_kinematic_particles(oracle_mod):
    model, cfg = lattice_scene((10, 10, 10), vel_std=0.1, device=DEV)
    n = model.particle_count
    rng = np.random.default_rng(5)
    flags = np.ones(n, np.int32)
    flags[rng.choice(n, 60, replace=False)] = 0
    kin = rng.choice(n, 40, replace=False)
    mass = model.particle_mass.cpu().numpy()
    mass[kin] = 0.0
    inv = np.divide(1.0, mass, out=np.zeros_like(mass), where=mass != 0).astype(np.float32)
    model.particle_flags.copy_(torch.from_numpy(flags))
    model.particle_mass.copy_(torch.from_numpy(mass))
    model.particle_inv_mass.copy_(torch.from_numpy(inv))
    from newton_sph_dev_b200.solvers import SolverSPH

    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    s1.particle_qd.fill_(-7.0)
    s0.particle_f.normal_(0, 1e-4)
    v_init = s1.particle_qd.cpu().numpy()
    solver.step(s0, s1, model.control(), None, 1e-4)
    torch.cuda.synchronize()
    h = _host(model, s0)
    r32 = _oracle_step(oracle_mod, solver, model, h, 1e-4, v_init, "f32")
    np.testing.assert_array_equal(s1.particle_q.cpu().numpy(), r32["x"])
    np.testing.assert_array_equal(s1.particle_qd.cpu().numpy(), r32["v"])
    off, ids = solver.neighbors()
    roff, rids = oracle_mod.sph_neighbors(cfg.constants(1e-4, 1e5)["f32"], solver.grid_dims, h["x"], flags)
    np.testing.assert_array_equal(ids.cpu().numpy(), rids)
    # inactive: position copied, velocity untouched
    ina = flags == 0
    assert np.array_equal(s1.particle_q.cpu().numpy()[ina], h["x"][ina])
    assert np.all(s1.particle_qd.cpu().numpy()[ina] == -7.0)


def test_100_steps_match_oracles(oracle_mod):
    """Dam break (32^3 lattice, spacing 0.01, 1 m box), 100 steps at dt = 1e-4."""
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg = lattice_scene((32, 32, 32), device=DEV, box_hi=(1.0, 1.0, 1.0), register=False)
    dt = 1e-4
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    h = _host(model, s0)
    x32, v32 = h["x"].copy(), h["v"].copy()
    x64, v64 = h["x"].astype(np.float64), h["v"].astype(np.float64)
    consts = cfg.constants(dt, model.particle_max_velocity)
    for _ in range(100):
        solver.step(s0, s1, None, None, dt)
        s0, s1 = s1, s0
        r = oracle_mod.sph_step(consts, solver.grid_dims, x32, v32, h["mass"], h["inv_mass"], h["flags"], h["world"],
                                h["gravity"], f_ext=h["f"], v_out_init=v32, precision="f32")
        x32, v32 = r["x"], r["v"]
        r = oracle_mod.sph_step(consts, solver.grid_dims, x64.astype(np.float32), v64.astype(np.float32), h["mass"],
                                h["inv_mass"], h["flags"], h["world"], h["gravity"], f_ext=h["f"],
                                v_out_init=v64, precision="f64")
        x64, v64 = r["x"], r["v"]
    torch.cuda.synchronize()
    xg = s0.particle_q.cpu().numpy()
    np.testing.assert_array_equal(xg, x32)
    np.testing.assert_array_equal(s0.particle_qd.cpu().numpy(), v32)
    # against fp64 (rounded to fp32 state between steps): 1e-3 of the box after 100 steps
    assert np.max(np.abs(xg.astype(np.float64) - x64)) < 1e-3 * 1.0
    assert solver.status() == 0


def test_free_fall_and_runtime_gravity():
    """newton/tests/test_runtime_gravity.py:18-67 with SolverSPH."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverNotifyFlags, SolverSPH

    b = nsph.ModelBuilder(gravity=-9.81)
    b.add_particle(pos=(0.0, 0.0, 1.0), vel=(0.0, 0.0, 0.0), mass=1.0)
    b.add_particle(pos=(5.0, 0.0, 1.0), vel=(0.0, 0.0, 0.0), mass=1.0)
    model = b.finalize(DEV)
    solver = SolverSPH(model, SolverSPH.Config(smoothing_length=0.1))
    s0, s1 = model.state(), model.state()
    control = model.control()
    dt = 0.01
    for _ in range(10):
        s0.clear_forces()
        solver.step(s0, s1, control, None, dt)
        s0, s1 = s1, s0
    vz = float(s0.particle_qd[0, 2])
    assert vz < -0.5 and abs(vz + 9.81 * 0.1) < 1e-4
    model.set_gravity((0.0, 0.0, 0.0))
    solver.notify_model_changed(SolverNotifyFlags.MODEL_PROPERTIES)
    for _ in range(10):
        solver.step(s0, s1, control, None, dt)
        s0, s1 = s1, s0
    assert abs(float(s0.particle_qd[0, 2]) - vz) < 1e-6
    model.set_gravity((0.0, 0.0, 9.81))
    for _ in range(20):
        solver.step(s0, s1, control, None, dt)
        s0, s1 = s1, s0
    assert float(s0.particle_qd[0, 2]) > vz


def test_graph_replay_sees_runtime_gravity():
    """newton/tests/test_runtime_gravity.py:141-210: a captured step reads the
    current gravity on replay."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    b = nsph.ModelBuilder(gravity=-9.81)
    for i in range(5):
        b.add_particle(pos=(i * 0.5, 0.0, 2.0), vel=(0.0, 0.0, 0.0), mass=1.0)
    model = b.finalize(DEV)
    solver = SolverSPH(model, SolverSPH.Config(smoothing_length=0.1))
    s0, s1 = model.state(), model.state()
    dt = 0.01
    solver.step(s0, s1, None, None, dt)  # warm-up outside the capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        solver.step(s0, s1, None, None, dt)
        solver.step(s1, s0, None, None, dt)
    for _ in range(5):
        graph.replay()
    torch.cuda.synchronize()
    v_def = float(s0.particle_qd[0, 2])
    assert v_def < -0.5
    model.set_gravity((0.0, 0.0, 0.0))
    for _ in range(5):
        graph.replay()
    torch.cuda.synchronize()
    assert abs(float(s0.particle_qd[0, 2]) - v_def) < 1e-5
    model.set_gravity((0.0, 0.0, 9.81))
    for _ in range(10):
        graph.replay()
    torch.cuda.synchronize()
    assert float(s0.particle_qd[0, 2]) > 0.5


def test_status_flags_and_errors():
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg = lattice_scene((6, 6, 6), device=DEV)
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, 1e-4)
    assert solver.status() == 0
    s0.particle_q[3, 1] = float("nan")
    solver.step(s0, s1, None, None, 1e-4)
    st = solver.status()
    assert st & 1  # NSPH_STATUS_NONFINITE_INPUT
    solver.reset_status()
    assert solver.status() == 0
    with pytest.raises(ValueError):
        solver.step(s0, s0, None, None, 1e-4)  # aliased in/out
    with pytest.raises(ValueError):
        solver.step(s0, s1, None, object(), 1e-4)  # contacts are not consumed


def test_integrate_particles_parity(oracle_mod):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverBase

    rng = np.random.default_rng(11)
    b = nsph.ModelBuilder()
    b.begin_world(gravity=(0.0, -3.0, 0.0))
    n = 5000
    b.add_particles(pos=rng.random((n, 3)), vel=rng.normal(0, 1, (n, 3)), mass=rng.random(n) + 0.1,
                    flags=(rng.random(n) > 0.1).astype(np.int32))
    b.end_world()
    b.add_particles(pos=rng.random((100, 3)), vel=rng.normal(0, 200, (100, 3)), mass=np.zeros(100))
    model = b.finalize(DEV)
    model.particle_max_velocity = 150.0
    s0, s1 = model.state(), model.state()
    s0.particle_f.normal_(0, 3)
    s1.particle_qd.fill_(-5.0)
    SolverBase(model).integrate_particles(model, s0, s1, 1e-3)
    torch.cuda.synchronize()
    h = _host(model, s0)
    xn = np.zeros_like(h["x"])
    vn = np.full_like(h["v"], -5.0)
    oracle_mod.integrate_particles(h["x"], h["v"], h["f"], h["inv_mass"], h["flags"], h["world"], h["gravity"],
                                   1e-3, 150.0, xn, vn)
    np.testing.assert_array_equal(s1.particle_q.cpu().numpy(), xn)
    np.testing.assert_array_equal(s1.particle_qd.cpu().numpy(), vn)


def test_full_size_tank_properties(oracle_mod):
    """1,048,576 particles (128x128x64 block, spacing 0.005, 2x1x1 m tank): the
    grid bit-exact against the oracle and size-independent checks of the
    step (neighbour counts, conservation of mass in the density sum,
    finiteness)."""
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg = lattice_scene((128, 128, 64), spacing=0.005, vel_std=0.01, device=DEV, box_hi=(2.0, 1.0, 1.0),
                               register=True)
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, 5e-5)
    torch.cuda.synchronize()
    x = s0.particle_q.cpu().numpy()
    consts = cfg.constants(5e-5, model.particle_max_velocity)
    g = solver.grid_arrays()
    ref = oracle_mod.grid_build(x, float(consts["f32"]["cell_width"]), solver.grid_dims)
    for k in ref:
        np.testing.assert_array_equal(g[k].cpu().numpy(), ref[k], err_msg=k)
    off, ids = solver.neighbors()
    roff, rids = oracle_mod.sph_neighbors(consts["f32"], solver.grid_dims, x, model.particle_flags.cpu().numpy())
    np.testing.assert_array_equal(off.cpu().numpy(), roff)
    np.testing.assert_array_equal(ids.cpu().numpy(), rids)
    rho = s1.sph.density.cpu().numpy()
    assert np.all(np.isfinite(s1.particle_q.cpu().numpy())) and np.all(np.isfinite(rho))
    # interior particles sit near rest density
    interior = (np.linalg.norm(x - x.mean(0), axis=1) < 0.15)
    assert abs(float(np.median(rho[interior])) - 1000.0) < 20.0
    assert solver.status() == 0


def test_launch_shape_does_not_change_results():
    """The autotuner may pick any launch shape: every shape gives the same bits."""
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg = lattice_scene((16, 12, 10), vel_std=0.1, device=DEV)
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, 1e-4)
    torch.cuda.synchronize()
    ref = (s1.particle_q.clone(), s1.particle_qd.clone(), s1.sph.density.clone())
    for shape in [(64, 0), (128, 1), (256, 4), (96, 2)]:
        solver.set_launch(*shape)
        solver.step(s0, s1, None, None, 1e-4)
        torch.cuda.synchronize()
        assert torch.equal(s1.particle_q, ref[0]) and torch.equal(s1.particle_qd, ref[1])
        assert torch.equal(s1.sph.density, ref[2])
    res = solver.autotune(s0, s1, 1e-4, candidates=[(128, 0), (256, 2)], repeats=1)
    assert res["best"] in [(128, 0), (256, 2)]
    solver.step(s0, s1, None, None, 1e-4)
    torch.cuda.synchronize()
    assert torch.equal(s1.particle_q, ref[0])
    with pytest.raises(ValueError):
        solver.set_launch(100, 0)
