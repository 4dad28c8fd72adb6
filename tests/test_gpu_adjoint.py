"""The hand-written adjoint on the GPU (nsph_sph_step_adjoint, sph_step,
sph_rollout): against the fp64 adjoint oracle on the same inputs, against
fp64 central finite differences (the pin of the gradient), checkpointing
invariance, determinism, and the reference's gradient-sign example
(newton/solvers.py:359-395, a wp.Tape over one step).

Tolerances. The device runs the step and its adjoint in fp32, the oracle in
fp64; device and fp64 gradients are compared by relative L2 error (measured
on a B200: below 1e-6 for one step and 1.2e-5 for a 20-step rollout):
<= 1e-4 for one step and <= 1e-3 for the rollout. Directional derivatives
against fp64 central differences (eps = 1e-3 in v0 and relative 1e-3 in B):
within 1e-4 without the pressure clamp; with it, within 1e-2, because a few
particles cross the clamp's kink at rho = rho0 inside the difference step
(measured 2.5e-3).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def block_scene(shape, s, seed, vel_std, box_hi=(1.0, 1.0, 1.0), clamp=True, v_max=None, n_inactive=0,
                n_kinematic=0, floor_shift=0.0, floor_speed=0.0):
    """A jittered lattice block as (model, config, x0, v0) with numpy copies."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in shape], indexing="ij"), -1).reshape(-1, 3)
    x = ((g + 0.5) * s + rng.uniform(-0.1 * s, 0.1 * s, g.shape)).astype(np.float32)
    x[:, 2] -= np.float32(floor_shift)
    v = rng.normal(0, vel_std, x.shape).astype(np.float32)
    v[:, 2] -= np.float32(floor_speed)
    n = len(x)
    b = nsph.ModelBuilder()
    b.add_particles(pos=x.tolist(), vel=v.tolist(), mass=[1000.0 * s**3] * n)
    model = b.finalize(DEV)
    if v_max is not None:
        model.particle_max_velocity = float(v_max)
    flags = np.ones(n, np.int32)
    if n_inactive:
        flags[rng.choice(n, n_inactive, replace=False)] = 0
    mass = model.particle_mass.cpu().numpy()
    inv = model.particle_inv_mass.cpu().numpy()
    if n_kinematic:
        inv[rng.choice(n, n_kinematic, replace=False)] = 0.0
    model.particle_flags.copy_(torch.from_numpy(flags))
    model.particle_inv_mass.copy_(torch.from_numpy(inv))
    cfg = SolverSPH.Config(smoothing_length=2 * s, box_lo=(0.0, 0.0, 0.0), box_hi=box_hi, clamp_pressure=clamp)
    return model, cfg, x, v, rng


def oracle_scene(oracle_mod, model, cfg, dt, f_ext=None):
    c64 = cfg.constants(dt, model.particle_max_velocity)["f64"]
    return oracle_mod.AdjScene(c64, model.particle_mass.cpu().numpy(), model.particle_inv_mass.cpu().numpy(),
                               model.particle_flags.cpu().numpy(), model.gravity.cpu().numpy(), f_ext=f_ext)


@pytest.mark.parametrize("clamp", [True, False])
def test_step_adjoint_matches_fp64_oracle(oracle_mod, clamp):
    """One step's VJP with every branch live: walls, |v| clamp, inactive and
    kinematic particles, external force, density adjoint."""
    from newton_sph_dev_b200.solvers import SolverSPH

    dt = 5e-4
    model, cfg, x, v, rng = block_scene((12, 10, 8), 0.01, 7, 0.3, clamp=clamp, v_max=1.5, n_inactive=9,
                                        n_kinematic=7, floor_shift=0.0046, floor_speed=1.0)
    n = len(x)
    solver = SolverSPH(model, cfg)
    f = (rng.normal(0, 1e-4, (n, 3))).astype(np.float32)
    xg1 = rng.normal(0, 1, (n, 3)).astype(np.float32)
    vg1 = rng.normal(0, 1e-3, (n, 3)).astype(np.float32)
    rg1 = rng.normal(0, 1e-6, n).astype(np.float32)
    T = lambda a: torch.from_numpy(a).to(DEV)
    xt, vt, ft = T(x), T(v), T(f)
    xg, vg, fg = torch.empty_like(xt), torch.empty_like(xt), torch.zeros_like(xt)
    bg = torch.zeros(1, device=DEV)
    solver.step_backward_raw(xt, vt, solver.step_params(dt), T(xg1), T(vg1), xg, vg, f_ext=ft,
                             rho_out_grad=T(rg1), f_ext_grad=fg, eos_b_grad=bg)
    torch.cuda.synchronize()
    sc = oracle_scene(oracle_mod, model, cfg, dt, f_ext=f)
    x1, v1, _ = oracle_mod.adj_step64(sc, x, v)
    act = model.particle_flags.cpu().numpy() != 0
    assert np.sum(x1[act, 2] <= 0.0) > 0, "no particle reached the floor"
    assert np.max(np.linalg.norm(v1[act], axis=1)) == pytest.approx(1.5), "|v| clamp not reached"
    rx, rv, rf, rb = oracle_mod.adj_vjp64(sc, x, v, xg1, vg1, rg1)
    errs = {"x": rel_l2(xg.cpu().numpy(), rx), "v": rel_l2(vg.cpu().numpy(), rv), "f": rel_l2(fg.cpu().numpy(), rf),
            "b": abs(float(bg.item()) - rb) / abs(rb)}
    print("step adjoint rel err vs fp64 oracle:", errs)
    assert max(errs.values()) <= 1e-4, errs
    # inactive particles pass their adjoints through
    ina = ~act
    np.testing.assert_array_equal(xg.cpu().numpy()[ina], xg1[ina])
    np.testing.assert_array_equal(vg.cpu().numpy()[ina], vg1[ina])


def test_adjoint_in_place_and_deterministic():
    """x_in_adj / v_in_adj may be the x_out_adj / v_out_adj buffers; repeated
    calls give identical bits."""
    from newton_sph_dev_b200.solvers import SolverSPH

    dt = 1e-4
    model, cfg, x, v, rng = block_scene((10, 10, 10), 0.01, 3, 0.1)
    solver = SolverSPH(model, cfg)
    n = len(x)
    xt, vt = torch.from_numpy(x).to(DEV), torch.from_numpy(v).to(DEV)
    xg1 = torch.from_numpy(rng.normal(0, 1, (n, 3)).astype(np.float32)).to(DEV)
    vg1 = torch.from_numpy(rng.normal(0, 1, (n, 3)).astype(np.float32)).to(DEV)
    p = solver.step_params(dt)
    outs = []
    for _ in range(2):
        xg, vg = torch.empty_like(xt), torch.empty_like(xt)
        bg = torch.zeros(1, device=DEV)
        solver.step_backward_raw(xt, vt, p, xg1, vg1, xg, vg, eos_b_grad=bg)
        outs.append((xg, vg, bg))
    xa, va = xg1.clone(), vg1.clone()
    bg = torch.zeros(1, device=DEV)
    solver.step_backward_raw(xt, vt, p, xa, va, xa, va, eos_b_grad=bg)
    torch.cuda.synchronize()
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)
    assert torch.equal(xa, outs[0][0]) and torch.equal(va, outs[0][1]) and torch.equal(bg, outs[0][2])


def _rollout_case(clamp):
    model, cfg, x, v, rng = block_scene((16, 16, 8), 0.01, 11, 0.1, clamp=clamp)
    y = (x + rng.normal(0, 0.01, x.shape)).astype(np.float32)
    return model, cfg, x, v, y, rng


@pytest.mark.parametrize("clamp", [False, True])
def test_rollout_gradient_matches_fp64_and_central_differences(oracle_mod, clamp):
    from newton_sph_dev_b200.solvers import SolverSPH, sph_rollout

    dt, steps = 1e-4, 20
    model, cfg, x, v, y, rng = _rollout_case(clamp)
    solver = SolverSPH(model, cfg)
    x0 = torch.from_numpy(x).to(DEV).requires_grad_(True)
    v0 = torch.from_numpy(v).to(DEV).requires_grad_(True)
    b = torch.tensor([float(solver.step_params(dt).eos_b)], device=DEV, requires_grad=True)
    yt = torch.from_numpy(y).to(DEV)
    xT, _ = sph_rollout(solver, x0, v0, steps, dt, eos_b=b, checkpoint_every=5)
    loss = ((xT - yt) ** 2).sum(dim=1).mean()
    loss.backward()
    gx, gv, gb = x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), float(b.grad.item())

    sc = oracle_scene(oracle_mod, model, cfg, dt)
    loss64, rx, rv, rb = oracle_mod.rollout_grad64(sc, x, v, steps, y)
    assert float(loss.item()) == pytest.approx(loss64, rel=1e-5)
    errs = {"x": rel_l2(gx, rx), "v": rel_l2(gv, rv), "b": abs(gb - rb) / abs(rb)}
    print(f"rollout gradient rel err vs fp64 adjoint (clamp={clamp}):", errs)
    assert max(errs.values()) <= 1e-3, errs

    # central differences of the fp64 rollout, eps = 1e-3 in v0
    B = sc.c64["eos_b"]
    tol = 1e-2 if clamp else 1e-4
    for trial in range(2):
        d = rng.normal(0, 1, x.shape)
        fd = (oracle_mod.mse_loss(oracle_mod.rollout64(sc, x, v + 1e-3 * d, steps)[0], y)
              - oracle_mod.mse_loss(oracle_mod.rollout64(sc, x, v - 1e-3 * d, steps)[0], y)) / 2e-3
        got = float(np.sum(gv * d))
        print(f"  v0 direction {trial}: fd {fd:.6e} device {got:.6e}")
        assert abs(got - fd) <= tol * abs(fd)
    fd = (oracle_mod.mse_loss(oracle_mod.rollout64(sc, x, v, steps, eos_b=B * (1 + 1e-3))[0], y)
          - oracle_mod.mse_loss(oracle_mod.rollout64(sc, x, v, steps, eos_b=B * (1 - 1e-3))[0], y)) / (2e-3 * B)
    print(f"  B: fd {fd:.6e} device {gb:.6e}")
    assert abs(gb - fd) <= tol * abs(fd)


def test_checkpointing_does_not_change_gradients():
    """Gradients are bit-identical for every checkpoint interval, and the
    un-checkpointed chain of sph_step nodes gives the same x0/v0 gradients."""
    from newton_sph_dev_b200.solvers import SolverSPH, sph_rollout, sph_step

    dt, steps = 1e-4, 12
    model, cfg, x, v, y, _ = _rollout_case(True)
    solver = SolverSPH(model, cfg)
    yt = torch.from_numpy(y).to(DEV)
    B0 = float(solver.step_params(dt).eos_b)

    def grads(every):
        x0 = torch.from_numpy(x).to(DEV).requires_grad_(True)
        v0 = torch.from_numpy(v).to(DEV).requires_grad_(True)
        b = torch.tensor([B0], device=DEV, requires_grad=True)
        if every is None:
            xt, vt = x0, v0
            for _ in range(steps):
                xt, vt = sph_step(solver, xt, vt, dt, eos_b=b)
        else:
            xt, vt = sph_rollout(solver, x0, v0, steps, dt, eos_b=b, checkpoint_every=every)
        (((xt - yt) ** 2).sum() + (vt ** 2).sum()).backward()
        return x0.grad, v0.grad, b.grad

    ref = grads(4)
    for every in (1, 5, steps, 100):
        g = grads(every)
        assert all(torch.equal(a, b) for a, b in zip(g, ref)), every
    g = grads(None)
    assert torch.equal(g[0], ref[0]) and torch.equal(g[1], ref[1])
    torch.testing.assert_close(g[2], ref[2], rtol=1e-5, atol=0)


def test_gradient_sign_like_the_reference_tape_example():
    """newton/solvers.py:359-395: one particle at the origin moving +x at
    1 m/s, one step of 1/60 s, loss |x - (0.25, 0, 0)|^2: the gradient of
    the loss with respect to the initial x-velocity is negative."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    b = nsph.ModelBuilder()
    b.add_particle(pos=(0.0, 0.0, 0.0), vel=(1.0, 0.0, 0.0), mass=1.0)
    model = b.finalize(DEV, requires_grad=True)
    solver = SolverSPH(model, SolverSPH.Config(smoothing_length=0.1))
    state_in, state_out = model.state(), model.state()
    state_in.clear_forces()
    solver.step(state_in, state_out, model.control(), None, 1.0 / 60.0)
    target = torch.tensor([0.25, 0.0, 0.0], device=DEV)
    loss = ((state_out.particle_q[0] - target) ** 2).sum()
    loss.backward()
    g = state_in.particle_qd.grad.cpu().numpy()
    assert float(g[0, 0]) < 0.0
    # analytic: x1 = x0 + (v0 + g dt) dt, so dL/dv0 = 2 (x1 - target) dt
    x1 = state_out.particle_q.detach().cpu().numpy()[0]
    expect = 2.0 * (x1 - target.cpu().numpy()) / 60.0
    np.testing.assert_allclose(g[0], expect, rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(state_in.particle_q.grad.cpu().numpy()[0], 2.0 * (x1 - target.cpu().numpy()),
                               rtol=1e-5, atol=1e-9)


def test_adjoint_argument_checks():
    from newton_sph_dev_b200 import _lib
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, _ = block_scene((4, 4, 4), 0.01, 0, 0.0)
    solver = SolverSPH(model, cfg)
    xt, vt = torch.from_numpy(x).to(DEV), torch.from_numpy(v).to(DEV)
    p = solver.step_params(1e-4)
    L = _lib.load()
    n = len(x)
    args = lambda xa, va, xo, vo: (solver._handle, __import__("ctypes").byref(p), n, xt.data_ptr(), vt.data_ptr(),
                                   None, model.particle_mass.data_ptr(), model.particle_inv_mass.data_ptr(),
                                   model.particle_flags.data_ptr(), model.particle_world.data_ptr(),
                                   model.gravity.data_ptr(), 1, xa, va, None, xo, vo, None, None,
                                   _lib.stream_handle(model.device))
    g1, g2 = torch.zeros_like(xt), torch.zeros_like(xt)
    # not enabled yet
    assert L.nsph_sph_step_adjoint(*args(g1.data_ptr(), g2.data_ptr(), g1.data_ptr(), g2.data_ptr())) == \
        _lib.NSPH_ERR_INVALID_ARG
    solver.enable_adjoint()
    assert L.nsph_sph_step_adjoint(*args(g1.data_ptr(), g2.data_ptr(), g1.data_ptr(), g2.data_ptr())) == _lib.NSPH_OK
    assert L.nsph_sph_step_adjoint(*args(None, g2.data_ptr(), g1.data_ptr(), g2.data_ptr())) == \
        _lib.NSPH_ERR_INVALID_ARG
    # position and velocity adjoints must not share memory
    assert L.nsph_sph_step_adjoint(*args(g1.data_ptr(), g2.data_ptr(), g2.data_ptr(), g1.data_ptr())) == \
        _lib.NSPH_ERR_INVALID_ARG
    torch.cuda.synchronize()
    with pytest.raises(ValueError):
        solver.step_backward_raw(xt, vt, p, g1[:5], g2, g1, g2)


def test_segment_tape_equals_recompute_then_reverse():
    """nsph_sph_segment_adjoint (recompute keeping each step's grid and
    density scratch, then reverse from it) is bit-identical to
    nsph_sph_rollout of the segment followed by nsph_sph_rollout_adjoint,
    with every branch live: walls, the |v| clamp, inactive and kinematic
    particles, an external force and the B gradient; and it leaves the
    solver's grid describing the segment's last input state."""
    from newton_sph_dev_b200.solvers import SolverSPH

    dt, steps = 1e-4, 7
    model, cfg, x, v, rng = block_scene((12, 12, 8), 0.01, 5, 0.3, v_max=0.5, n_inactive=17, n_kinematic=13,
                                        floor_shift=0.004, floor_speed=0.5)
    solver = SolverSPH(model, cfg)
    n = len(x)
    p = solver.step_params(dt)
    x0, v0 = torch.from_numpy(x).to(DEV), torch.from_numpy(v).to(DEV)
    f = torch.from_numpy(rng.normal(0, 1e-3, x.shape).astype(np.float32)).to(DEV)
    gx = torch.from_numpy(rng.normal(0, 1, x.shape).astype(np.float32)).to(DEV)
    gv = torch.from_numpy(rng.normal(0, 1, x.shape).astype(np.float32)).to(DEV)

    # recompute, then reverse
    sx = torch.empty((steps, n, 3), dtype=torch.float32, device=DEV)
    sv = torch.empty_like(sx)
    sx[0].copy_(x0)
    sv[0].copy_(v0)
    solver.rollout_raw(sx[0], sv[0], sx[1:], sv[1:], p, f)
    xa, va = gx.clone(), gv.clone()
    fa, ba = torch.zeros_like(x0), torch.zeros(1, device=DEV)
    solver.rollout_backward_raw(sx, sv, p, xa, va, f_ext=f, f_ext_grad=fa, eos_b_grad=ba)

    # the tape
    xb, vb = gx.clone(), gv.clone()
    fb, bb = torch.zeros_like(x0), torch.zeros(1, device=DEV)
    solver.segment_backward_raw(x0, v0, steps, p, xb, vb, f_ext=f, f_ext_grad=fb, eos_b_grad=bb)
    torch.cuda.synchronize()
    assert torch.isfinite(xa).all() and float(xa.abs().max()) > 0.0
    for a, b in ((xa, xb), (va, vb), (fa, fb), (ba, bb)):
        assert torch.equal(a, b)
    assert solver.status() == 0

    # the solver's grid and mirrors now describe the last input state: its
    # neighbour lists equal those of a plain step on that state
    after = solver.neighbors()
    solver.step_raw(sx[steps - 1], sv[steps - 1], torch.empty_like(x0), sv[steps - 1].clone(), p, f)
    ref = solver.neighbors()
    assert all(torch.equal(a, b) for a, b in zip(after, ref))

    # a longer segment than the tape holds grows it; a shorter one reuses it
    xc, vc = gx.clone(), gv.clone()
    solver.segment_backward_raw(x0, v0, 2, p, xc, vc, f_ext=f)
    solver.segment_backward_raw(x0, v0, steps + 3, p, xc, vc, f_ext=f)
    torch.cuda.synchronize()
    assert torch.isfinite(xc).all()


def test_segment_adjoint_argument_checks():
    import ctypes

    from newton_sph_dev_b200 import _lib
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, _ = block_scene((4, 4, 4), 0.01, 0, 0.0)
    solver = SolverSPH(model, cfg)
    xt, vt = torch.from_numpy(x).to(DEV), torch.from_numpy(v).to(DEV)
    p = solver.step_params(1e-4)
    L = _lib.load()
    n = len(x)

    def call(x0, v0, xa, va, steps=3):
        return L.nsph_sph_segment_adjoint(solver._handle, ctypes.byref(p), n, steps, x0, v0, None,
                                          model.particle_mass.data_ptr(), model.particle_inv_mass.data_ptr(),
                                          model.particle_flags.data_ptr(), model.particle_world.data_ptr(),
                                          model.gravity.data_ptr(), 1, xa, va, None, None,
                                          _lib.stream_handle(model.device))

    g1, g2 = torch.zeros_like(xt), torch.zeros_like(xt)
    # adjoint scratch not enabled yet
    assert call(xt.data_ptr(), vt.data_ptr(), g1.data_ptr(), g2.data_ptr()) == _lib.NSPH_ERR_INVALID_ARG
    solver.enable_adjoint()
    assert call(xt.data_ptr(), vt.data_ptr(), g1.data_ptr(), g2.data_ptr()) == _lib.NSPH_OK
    assert call(xt.data_ptr(), vt.data_ptr(), None, g2.data_ptr()) == _lib.NSPH_ERR_INVALID_ARG
    # adjoints overlapping each other or the initial state
    assert call(xt.data_ptr(), vt.data_ptr(), g1.data_ptr(), g1.data_ptr()) == _lib.NSPH_ERR_INVALID_ARG
    assert call(xt.data_ptr(), vt.data_ptr(), xt.data_ptr(), g2.data_ptr()) == _lib.NSPH_ERR_INVALID_ARG
    assert call(xt.data_ptr(), vt.data_ptr(), g1.data_ptr(), g2.data_ptr(), steps=-1) == _lib.NSPH_ERR_INVALID_ARG
    assert call(xt.data_ptr(), vt.data_ptr(), g1.data_ptr(), g2.data_ptr(), steps=0) == _lib.NSPH_OK
    assert L.nsph_sph_reserve_segment(solver._handle, -1) == _lib.NSPH_ERR_INVALID_ARG
    torch.cuda.synchronize()
    with pytest.raises(ValueError):
        solver.segment_backward_raw(xt, vt, 2, p, g1[:5], g2)
