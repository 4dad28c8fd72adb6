"""Host-side pieces of the surrogate step (CPU only): the fp64 restatement of
the neighbour features against the fp64 oracle step, the training-target
algebra, and the fallback rule of the stepper."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from newton_sph_dev_b200.solvers.sph import SPHConfig
from newton_sph_dev_b200.solvers.sph_surrogate import FallbackMonitor, accel_scale, surrogate_targets


def _block(shape, s, seed, vel):
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in shape], indexing="ij"), -1).reshape(-1, 3)
    x = ((g + 0.5) * s + rng.uniform(-0.1 * s, 0.1 * s, g.shape)).astype(np.float32)
    v = rng.normal(0, vel, x.shape).astype(np.float32)
    return x, v


def test_feature_restatement_matches_fp64_step(oracle_mod):
    s = 0.01
    x, v = _block((9, 8, 7), s, 5, 0.2)
    n = len(x)
    cfg = SPHConfig(smoothing_length=2 * s, box_lo=(0, 0, 0), box_hi=(0.5, 0.5, 0.5))
    consts = cfg.constants(4e-4, 1e5)
    m = np.full(n, 1000 * s**3, np.float32)
    flags = np.ones(n, np.int32)
    flags[:5] = 0
    f, rho, a, dv = oracle_mod.surrogate_features_py(consts, cfg.resolved_grid_dims(), x, v, m, flags)
    ref = oracle_mod.sph_step(consts, cfg.resolved_grid_dims(), x, v, m, (1 / m).astype(np.float32), flags,
                              np.zeros(n, np.int32), np.array([[0, 0, -9.81]], np.float32), v_out_init=v,
                              precision="f64")
    np.testing.assert_allclose(rho, ref["rho"], rtol=1e-12)
    np.testing.assert_allclose(a, ref["a"], rtol=1e-9, atol=1e-9 * np.abs(ref["a"]).max())
    assert np.all(f[:5] == 0)
    # interior particles of a near-rest lattice (two spacings from the block's
    # faces): Shepard sum ~ 1, density ~ rho0
    act = flags != 0
    gi = np.stack(np.meshgrid(*[np.arange(k) for k in (9, 8, 7)], indexing="ij"), -1).reshape(-1, 3)
    inner = act & np.all((gi >= 2) & (gi <= np.array([9, 8, 7]) - 3), axis=1)
    assert inner.sum() > 20
    assert np.all(np.abs(f[inner, 0] - 1) < 0.1)
    assert np.all(np.abs(f[inner, 12] - 1) < 0.1)
    np.testing.assert_allclose(f[:, 1], f[:, 0] - 1 * act, atol=1e-15)
    np.testing.assert_allclose(f[:, 15], np.linalg.norm(f[:, 8:11], axis=1), rtol=1e-12)


def test_surrogate_targets_reproduce_the_landing_point():
    """With the target correction, one big step lands exactly where the
    reference trajectory landed."""
    cfg = SPHConfig(smoothing_length=0.02, box_lo=(0, 0, 0), box_hi=(1, 1, 1), xsph=0.01)
    g = torch.Generator().manual_seed(0)
    n, dt = 500, 4e-4
    x0 = torch.rand((n, 3), generator=g, dtype=torch.float64) * 0.5 + 0.25
    v0 = torch.randn((n, 3), generator=g, dtype=torch.float64) * 0.2
    x1 = x0 + v0 * dt + torch.randn((n, 3), generator=g, dtype=torch.float64) * 1e-6
    acc = torch.randn((n, 6), generator=g, dtype=torch.float64)
    grav = torch.tensor([0.0, 0.0, -9.81], dtype=torch.float64)
    target, ok = surrogate_targets(cfg, dt, x0, v0, x1, acc, grav)
    assert bool(ok.all())
    da = target * accel_scale(cfg)
    v1 = v0 + (acc[:, :3] + da + grav) * dt + cfg.xsph * acc[:, 3:]
    torch.testing.assert_close(x0 + v1 * dt, x1, rtol=0, atol=1e-13)
    # rows that end on or outside a wall are not usable
    x1b = x1.clone()
    x1b[0, 2] = 0.0
    _, ok = surrogate_targets(cfg, dt, x0, v0, x1b, acc, grav)
    assert not bool(ok[0]) and bool(ok[1:].all())


def test_accel_scale_is_c0_squared_over_h():
    cfg = SPHConfig(smoothing_length=0.01, sound_speed=20.0)
    assert accel_scale(cfg) == pytest.approx(400.0 / 0.01, rel=1e-6)


def test_fallback_monitor():
    m = FallbackMonitor(threshold=0.01, cooldown=2)
    assert m.use_surrogate()
    m.end_window(0.005)
    assert m.use_surrogate() and m.trips == 0
    m.end_window(0.02)  # trip: two plain windows follow
    assert not m.use_surrogate() and m.trips == 1
    m.end_window(None)
    assert not m.use_surrogate()
    m.end_window(None)
    assert m.use_surrogate()
    m.end_window(math.nan)  # a non-finite monitor value trips too
    assert not m.use_surrogate() and m.trips == 2


def test_fallback_monitor_backoff():
    """With backoff, each failure in a row doubles the suspension (capped);
    a window that passes resets it."""
    m = FallbackMonitor(threshold=0.01, cooldown=1, backoff=True, max_cooldown=4)

    def plain_windows():
        k = 0
        while not m.use_surrogate():
            m.end_window(None)
            k += 1
        return k

    assert m.end_window(0.5) is True
    assert plain_windows() == 1
    assert m.end_window(0.5) is True
    assert plain_windows() == 2
    assert m.end_window(math.nan) is True
    assert plain_windows() == 4
    assert m.end_window(0.5) is True
    assert plain_windows() == 4  # capped
    assert m.end_window(0.001) is False  # passes: the next failure starts over
    assert m.end_window(0.5) is True
    assert plain_windows() == 1
    assert m.trips == 5
