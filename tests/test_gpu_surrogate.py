"""The surrogate step on the GPU: the tcgen05 MLP kernels against a plain
torch fp32 reference of the same network, the hand-written training
gradient against torch autograd, the neighbour-feature pass against the fp64
restatement, and the surrogate step with a zero correction against the plain
step (bit for bit).

Tolerances. The MLP runs with bf16 weights and activations and fp32
accumulation; the reference rounds at the same places, but its SiLU is exact
where the kernel uses the tanh.approx instruction, and its sums run in
another order, so a hidden activation can round to the neighbouring bf16
value. Outputs are compared within 1e-2 of the output scale (measured on a
B200: 2.6e-3); the gradient by relative L2 error within 2e-3 (measured
2.5e-4), each parameter block within 1e-2. Features: fp32 sums against fp64, within
1e-4 of each feature's range (the acceleration features within 1e-3, as
the Tait EOS amplifies density rounding); the SPH acceleration the feature
pass returns is bit-exact with the fp32 oracle.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def random_model(seed=0, norm=True):
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel

    m = SurrogateModel(DEV, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    m.buf[1024:1088] = (torch.randn(64, generator=g) * 0.1).to(DEV)  # b1
    m.buf[5184:5248] = (torch.randn(64, generator=g) * 0.1).to(DEV)  # b2
    m.buf[5440:5443] = (torch.randn(3, generator=g) * 0.1).to(DEV)  # b3
    if norm:
        m.set_normalization(torch.randn(16, generator=g), torch.rand(16, generator=g) + 0.5,
                            torch.randn(3, generator=g), torch.rand(3, generator=g) + 0.5)
    return m


def test_mlp_forward_matches_torch_reference():
    m = random_model(0)
    g = torch.Generator().manual_seed(3)
    for n in (1, 127, 1000, 70001):  # ragged tails, several tiles per CTA
        f = (torch.randn((n, 16), generator=g) * 1.5 + 0.3).to(DEV)
        out = m.forward(f)
        ref = m.reference_forward(f)
        torch.cuda.synchronize()
        scale = float(ref.abs().max())
        err = float((out - ref).abs().max())
        print(f"n={n}: max |out - ref| = {err:.3e}, max |ref| = {scale:.3e}")
        assert err <= 1e-2 * scale, (n, err, scale)
        assert torch.isfinite(out).all()


def _autograd_reference(model, feat, target, idx):
    """Loss and gradient of the kernels' network in torch fp32: bf16 roundings
    of inputs, weights and hidden activations pass gradients straight through."""
    bf = lambda t: t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()
    buf = model.buf.detach().clone().requires_grad_(True)
    w1, b1 = buf[0:1024].view(16, 64), buf[1024:1088]
    w2, b2 = buf[1088:5184].view(64, 64), buf[5184:5248]
    w3, b3 = buf[5248:5440].view(64, 3), buf[5440:5443]
    f = feat[idx.long()]
    t = target[idx.long()]
    x = bf((f - buf[5448:5464]) * buf[5464:5480]).detach()
    h1 = bf(torch.nn.functional.silu(x @ bf(w1) + b1))
    h2 = bf(torch.nn.functional.silu(h1 @ bf(w2) + b2))
    y = h2 @ bf(w3) + b3
    tn = (t - buf[5480:5483].detach()) / buf[5484:5487].detach()
    loss = ((y - tn) ** 2).mean()
    loss.backward()
    return float(loss.detach()), buf.grad[:5443]


def test_mlp_gradient_matches_autograd():
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateTrainer

    m = random_model(1)
    g = torch.Generator().manual_seed(4)
    N = 5000
    feat = (torch.randn((N, 16), generator=g) * 1.5).to(DEV)
    target = (torch.randn((N, 3), generator=g)).to(DEV)
    for batch in (300, 4096):
        idx = torch.randint(0, N, (batch,), generator=g).to(DEV)
        tr = SurrogateTrainer(m)
        grad = tr.gradient(feat, target, idx).clone()
        torch.cuda.synchronize()
        ref_loss, ref_grad = _autograd_reference(m, feat, target, idx)
        rel = float((grad[:5443] - ref_grad).norm() / ref_grad.norm())
        print(f"batch {batch}: loss {float(grad[5443]):.6f} vs {ref_loss:.6f}, grad rel L2 {rel:.3e}")
        assert float(grad[5443]) == pytest.approx(ref_loss, rel=1e-3)
        assert rel <= 2e-3
        # each block of the gradient separately (W1, b1, W2, b2, W3, b3)
        for a, b in ((0, 1024), (1024, 1088), (1088, 5184), (5184, 5248), (5248, 5440), (5440, 5443)):
            r = float((grad[a:b] - ref_grad[a:b]).norm() / ref_grad[a:b].norm().clamp_min(1e-12))
            assert r <= 1e-2, (a, b, r)
        assert tr.err.item() == 0


def test_training_reduces_the_loss():
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel, train

    g = torch.Generator().manual_seed(5)
    N = 200000
    feat = torch.randn((N, 16), generator=g)
    w = torch.randn((16, 3), generator=g) * 0.3
    target = torch.tanh(feat @ w) + 0.1 * feat[:, :3] ** 2
    m = SurrogateModel(DEV, seed=2)
    res = train(m, feat.to(DEV), target.to(DEV), iters=300, batch=8192, lr=3e-3, log_every=50)
    print("training:", res["history"], "val", res["val_loss"])
    assert res["history"][0][1] > 0.5
    assert res["val_loss"] < 0.2 * res["history"][0][1]


def _scene(shape=(14, 13, 12), s=0.01, seed=3, vel=0.2):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    rng = np.random.default_rng(seed)
    gi = np.stack(np.meshgrid(*[np.arange(k) for k in shape], indexing="ij"), -1).reshape(-1, 3)
    x = ((gi + 0.5) * s + rng.uniform(-0.1 * s, 0.1 * s, gi.shape)).astype(np.float32)
    v = rng.normal(0, vel, x.shape).astype(np.float32)
    n = len(x)
    b = nsph.ModelBuilder()
    b.add_particles(pos=x.tolist(), vel=v.tolist(), mass=[1000.0 * s**3] * n)
    model = b.finalize(DEV)
    flags = np.ones(n, np.int32)
    flags[rng.choice(n, 11, replace=False)] = 0
    model.particle_flags.copy_(torch.from_numpy(flags))
    cfg = SolverSPH.Config(smoothing_length=2 * s, box_lo=(0.0, 0.0, 0.0), box_hi=(0.5, 0.5, 0.5))
    return model, cfg, x, v, flags


def test_features_match_fp64_restatement(oracle_mod):
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene()
    n = len(x)
    solver = SolverSPH(model, cfg)
    dt = 4e-4
    feat = torch.empty((n, 16), device=DEV)
    acc = torch.empty((n, 6), device=DEV)
    rho = torch.empty(n, device=DEV)
    solver.features_raw(model.particle_q, model.particle_qd, feat, acc, rho, params=solver.step_params(dt))
    torch.cuda.synchronize()
    consts = cfg.constants(dt, model.particle_max_velocity)
    dims = cfg.resolved_grid_dims()
    ref, _, _, _ = oracle_mod.surrogate_features_py(consts, dims, x, v, model.particle_mass.cpu().numpy(), flags)
    got = feat.cpu().numpy()
    for k in range(16):
        rng_k = max(np.abs(ref[:, k]).max(), 1e-12)
        tol = 1e-3 if k in (8, 9, 10, 14, 15) else 1e-4
        err = np.abs(got[:, k] - ref[:, k]).max() / rng_k
        assert err <= tol, (k, err)
    # the SPH acceleration and density are the plain step's, bit for bit
    r32 = oracle_mod.sph_step(consts, dims, x, v, model.particle_mass.cpu().numpy(),
                              model.particle_inv_mass.cpu().numpy(), flags, np.zeros(n, np.int32),
                              model.gravity.cpu().numpy(), v_out_init=v, precision="f32")
    np.testing.assert_array_equal(acc.cpu().numpy()[:, :3], r32["a"])
    np.testing.assert_array_equal(rho.cpu().numpy(), r32["rho"])


def test_zero_correction_is_the_plain_step_and_monitor():
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel, accel_scale

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=8)
    n = len(x)
    solver = SolverSPH(model, cfg)
    m = SurrogateModel(DEV, seed=0)
    m.zero_correction()
    dt = 4e-4
    p = solver.step_params(dt)
    stats = torch.zeros(4, device=DEV)
    xs, vs = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, xs, vs, p, m, accel_scale(cfg), stats)
    xp, vp = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_raw(model.particle_q, model.particle_qd, xp, vp, p)
    torch.cuda.synchronize()
    assert torch.equal(xs, xp) and torch.equal(vs, vp)
    # the compression monitor of that step
    rho = torch.empty(n, device=DEV)
    solver.features_raw(model.particle_q, model.particle_qd, rho_out=rho, params=p)
    act = torch.from_numpy(flags != 0).to(DEV)
    e = torch.clamp(rho[act] / 1000.0 - 1.0, min=0).mean()
    s = stats.cpu()
    assert float(s[0]) == pytest.approx(float(e), rel=1e-5, abs=1e-9)
    assert float(s[1]) == float(s[0]) and float(s[2]) == 1.0 and float(s[3]) == float(s[0])
    assert solver.status() == 0


def test_stepper_fallback_runs_plain_substeps():
    """Without rollback, a threshold below any possible error trips the
    monitor after the first window, which is kept: the next window runs plain
    substeps, bit-identical to a rollout of plain steps."""
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel, SurrogateSPH

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=9)
    solver = SolverSPH(model, cfg)
    m = SurrogateModel(DEV, seed=0)
    m.zero_correction()
    st = SurrogateSPH(solver, m, substeps=4, threshold=-1.0, window=2, cooldown=1, rollback=False, backoff=False)
    s0, s1 = model.state(), model.state()
    dt = 1e-4
    for _ in range(2):  # window 1: surrogate
        st.step(s0, s1, dt)
        s0, s1 = s1, s0
    assert st.surrogate_steps == 2 and st.monitor.trips == 1
    ref_x, ref_v = s0.particle_q.clone(), s0.particle_qd.clone()
    st.step(s0, s1, dt)  # window 2: plain substeps
    assert st.fallback_calls == 1
    tx = torch.empty((4, model.particle_count, 3), device=DEV)
    tv = torch.empty_like(tx)
    solver.rollout_raw(ref_x, ref_v, tx, tv, solver.step_params(dt))
    torch.cuda.synchronize()
    assert torch.equal(s1.particle_q, tx[-1]) and torch.equal(s1.particle_qd, tv[-1])
    st.step(s1, s0, dt)
    st.step(s0, s1, dt)  # window 3: surrogate again (cooldown over)
    assert st.surrogate_steps == 3 and st.fallback_calls == 2


def test_stepper_rollback_replaces_failed_window():
    """With rollback (the default), a failed window is replaced: the call that
    ends it returns the plain trajectory from the window's starting state,
    bit for bit, the window's surrogate steps are not counted, and the
    suspensions after consecutive failures grow (1, then 2 windows)."""
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateSPH

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=13)
    solver = SolverSPH(model, cfg)
    m = random_model(7)
    st = SurrogateSPH(solver, m, substeps=4, threshold=-1.0, window=2, cooldown=1)
    s0, s1 = model.state(), model.state()
    dt = 1e-4
    x0, v0 = s0.particle_q.clone(), s0.particle_qd.clone()
    for _ in range(2):  # window 1: surrogate, rejected
        st.step(s0, s1, dt)
        s0, s1 = s1, s0
    assert st.rollbacks == 1 and st.surrogate_steps == 0 and st.fallback_calls == 2
    tx = torch.empty((8, model.particle_count, 3), device=DEV)
    tv = torch.empty_like(tx)
    solver.rollout_raw(x0, v0, tx, tv, solver.step_params(dt))
    torch.cuda.synchronize()
    assert torch.equal(s0.particle_q, tx[-1]) and torch.equal(s0.particle_qd, tv[-1])
    modes = []
    for _ in range(10):  # plain (1 window), surrogate (rejected), plain (2 windows), surrogate
        before = st.surrogate_steps + st.rollbacks * 2
        st.step(s0, s1, dt)
        s0, s1 = s1, s0
        modes.append("s" if st.surrogate_steps + st.rollbacks * 2 > before else "p")
    assert "".join(modes) == "ppssppppss"
    assert st.rollbacks == 3 and st.mean_compression() == 0.0
    assert bool(torch.isfinite(s0.particle_q).all())


def test_fallback_trips_on_corrupted_weights():
    """Weights corrupted on the host (an output offset that drives every
    particle down at about 500 g) compress the block against the floor: the
    real 1% threshold trips the monitor, and the next window runs plain
    substeps."""
    from newton_sph_dev_b200.solvers.sph_surrogate import OUT_MEAN, SurrogateModel, SurrogateSPH, accel_scale

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=10)
    solver = SolverSPH(model, cfg)
    m = SurrogateModel(DEV, seed=0)
    m.zero_correction()
    m.buf[OUT_MEAN + 2] = -500.0 * 9.81 / accel_scale(cfg)  # the injected fault
    st = SurrogateSPH(solver, m, substeps=4, threshold=0.01, window=4, cooldown=1)
    s0, s1 = model.state(), model.state()
    dt = 1e-4
    for _ in range(4):
        st.step(s0, s1, dt)
        s0, s1 = s1, s0
    # tripped, and the window was replaced by plain steps (no compression left)
    assert st.monitor.trips == 1 and st.window_worst[-1] > 0.01 and st.rollbacks == 1
    assert st.fallback_calls == 4 and st.surrogate_steps == 0
    rho = torch.empty(model.particle_count, device=DEV)
    solver.features_raw(s0.particle_q, s0.particle_qd, rho_out=rho, params=solver.step_params(dt))
    assert float(torch.clamp(rho / 1000.0 - 1.0, min=0).mean()) < 0.01
    st.step(s0, s1, dt)
    assert st.fallback_calls == 5


def test_surrogate_wait_timeout_falls_back():
    """MMA-completion waits that give up at once (wait limit 0): the step
    integrates without the correction (the plain step at this dt, bit for
    bit), sets NSPH_STATUS_SURROGATE_TIMEOUT, and the stepper counts the
    window as failed and falls back."""
    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateSPH

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=11)
    solver = SolverSPH(model, cfg)
    m = random_model(5)
    solver.set_surrogate_wait_limit(0)
    dt = 1e-4
    p = solver.step_params(4 * dt)
    stats = torch.zeros(4, device=DEV)
    xs, vs = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, xs, vs, p, m, 1.0, stats)
    xp, vp = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_raw(model.particle_q, model.particle_qd, xp, vp, p)
    torch.cuda.synchronize()
    assert solver.status() & 8  # NSPH_STATUS_SURROGATE_TIMEOUT
    assert torch.equal(xs, xp) and torch.equal(vs, vp)
    solver.reset_status()
    st = SurrogateSPH(solver, m, substeps=4, threshold=0.01, window=2, cooldown=1)
    s0, s1 = model.state(), model.state()
    for _ in range(2):
        st.step(s0, s1, dt)
        s0, s1 = s1, s0
    assert st.timeouts == 1 and st.monitor.trips == 1 and st.rollbacks == 1
    st.step(s0, s1, dt)
    assert st.fallback_calls == 3
    solver.set_surrogate_wait_limit(-1)  # the default again: the corrected step runs
    solver.reset_status()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, xs, vs, p, m, 1.0, stats)
    torch.cuda.synchronize()
    assert solver.status() == 0
    assert not torch.equal(xs, xp)


@pytest.mark.parametrize("ctas_per_sm,tiles_per_cta", [(1, 1), (2, 1), (4, 1), (0, 2), (1, 2), (2, 2)])
def test_surrogate_launch_shape_keeps_results(ctas_per_sm, tiles_per_cta):
    """Other launch shapes of the fused kernel (fewer resident CTAs per SM, a
    larger L1 for its gathers; two tiles per CTA sharing the weights): the
    same positions and velocities, bit for bit, as the default launch, and
    the same compression statistics up to the order of the per-CTA partial
    sums."""
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=12)
    solver = SolverSPH(model, cfg)
    m = random_model(6)
    p = solver.step_params(4e-4)
    out = []
    for k, t in ((0, 0), (ctas_per_sm, tiles_per_cta)):
        solver.set_surrogate_launch(k, t)
        stats = torch.zeros(4, device=DEV)
        xs, vs = torch.empty_like(model.particle_q), model.particle_qd.clone()
        solver.step_surrogate_raw(model.particle_q, model.particle_qd, xs, vs, p, m, 1.0, stats)
        torch.cuda.synchronize()
        out.append((xs, vs, stats))
    solver.set_surrogate_launch(0)
    assert solver.status() == 0
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    torch.testing.assert_close(out[0][2], out[1][2], rtol=1e-5, atol=0.0)


def test_grouped_surrogate_wait_timeout_is_the_plain_step():
    """Two tiles per CTA with waits that give up at once: each group
    integrates without the correction (the plain step at this dt, bit for
    bit) and the status bit is set; the default limit again gives the
    corrected step, as the one-tile kernel does."""
    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, x, v, flags = _scene(seed=14)
    solver = SolverSPH(model, cfg)
    m = random_model(8)
    solver.set_surrogate_launch(0, 2)
    solver.set_surrogate_wait_limit(0)
    p = solver.step_params(4e-4)
    stats = torch.zeros(4, device=DEV)
    xs, vs = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, xs, vs, p, m, 1.0, stats)
    xp, vp = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_raw(model.particle_q, model.particle_qd, xp, vp, p)
    torch.cuda.synchronize()
    assert solver.status() & 8
    assert torch.equal(xs, xp) and torch.equal(vs, vp)
    solver.reset_status()
    solver.set_surrogate_wait_limit(-1)
    x1, v1 = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, x1, v1, p, m, 1.0, stats)
    solver.set_surrogate_launch(0, 1)
    x2, v2 = torch.empty_like(model.particle_q), model.particle_qd.clone()
    solver.step_surrogate_raw(model.particle_q, model.particle_qd, x2, v2, p, m, 1.0, stats)
    solver.set_surrogate_launch(0, 0)
    torch.cuda.synchronize()
    assert solver.status() == 0
    assert torch.equal(x1, x2) and torch.equal(v1, v2) and not torch.equal(x1, xp)
