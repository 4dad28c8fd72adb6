"""The fp32 restatement of the reference's particle-particle contact kernels
(oracle/contact.c): known answers of the force law (eval_particle_contact /
particle_force, newton/_src/solvers/semi_implicit/kernels_contact.py:11-84)
and of the XPBD correction (solve_particle_particle_contacts,
newton/_src/solvers/xpbd/kernels.py:225-289), and a brute-force O(N^2) fp64
restatement that pins the grid query. CPU only."""

from __future__ import annotations

import numpy as np
import pytest

DIMS = (128, 128, 128)
KE, KD, KF, MU = 1000.0, 100.0, 100.0, 0.5


def forces(O, x, v, r, flags=None, cohesion=0.0, grid_radius=None, f_init=None):
    x = np.asarray(x, np.float32)
    n = len(x)
    flags = np.ones(n, np.int32) if flags is None else flags
    rmax = float(np.max(r))
    return O.particle_contact_forces(x, np.asarray(v, np.float32), np.asarray(r, np.float32), flags,
                                     grid_radius or 2 * rmax + cohesion, DIMS, KE, KD, KF, MU, cohesion, rmax,
                                     f_init=f_init)


def test_normal_force_and_damping(oracle_mod):
    x = [[0.0, 0.0, 0.0], [0.15, 0.0, 0.0]]
    r = [0.1, 0.1]
    f = forces(oracle_mod, x, np.zeros((2, 3)), r)
    np.testing.assert_allclose(f, [[-50.0, 0, 0], [50.0, 0, 0]], rtol=1e-6)
    # approaching at 1 m/s: damping adds min(vn, 0) kd = -100 to fn
    v = [[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]]
    f = forces(oracle_mod, x, v, r)
    np.testing.assert_allclose(f, [[-150.0, 0, 0], [150.0, 0, 0]], rtol=1e-6)
    # separating: no damping term
    f = forces(oracle_mod, x, -np.asarray(v), r)
    np.testing.assert_allclose(f, [[-50.0, 0, 0], [50.0, 0, 0]], rtol=1e-6)


def test_friction_is_coulomb_limited(oracle_mod):
    x = [[0.0, 0.0, 0.0], [0.15, 0.0, 0.0]]
    r = [0.1, 0.1]
    # slow sliding: friction = |vt| kf = 0.2 * 100 = 20 < mu |fn| = 25, opposing the relative motion
    v = [[0.0, 0.1, 0.0], [0.0, -0.1, 0.0]]
    f = forces(oracle_mod, x, v, r)
    np.testing.assert_allclose(f[0], [-50.0, -20.0, 0.0], rtol=1e-6)
    # fast sliding: capped at mu |fn| = 25
    v = [[0.0, 1.0, 0.0], [0.0, -1.0, 0.0]]
    f = forces(oracle_mod, x, v, r)
    np.testing.assert_allclose(f[0], [-50.0, -25.0, 0.0], rtol=1e-6)


def test_cohesion_range(oracle_mod):
    r = [0.1, 0.1]
    x = [[0.0, 0.0, 0.0], [0.21, 0.0, 0.0]]  # gap 0.01
    f = forces(oracle_mod, x, np.zeros((2, 3)), r, cohesion=0.02)
    np.testing.assert_allclose(f[0], [10.0, 0.0, 0.0], rtol=1e-5)  # err = +0.01: attraction
    f = forces(oracle_mod, x, np.zeros((2, 3)), r, cohesion=0.005)
    np.testing.assert_array_equal(f, np.zeros((2, 3)))


def test_inactive_particles_are_skipped_and_not_written(oracle_mod):
    x = [[0.0, 0.0, 0.0], [0.15, 0.0, 0.0], [0.0, 0.15, 0.0]]
    r = [0.1, 0.1, 0.1]
    flags = np.array([1, 0, 1], np.int32)
    init = np.full((3, 3), 7.0, np.float32)
    f = forces(oracle_mod, x, np.zeros((3, 3)), r, flags=flags, f_init=init)
    np.testing.assert_array_equal(f[1], [7.0, 7.0, 7.0])
    np.testing.assert_allclose(f[0], [0.0, -50.0, 0.0], rtol=1e-6)


def test_xpbd_deltas(oracle_mod):
    O = oracle_mod
    x = np.array([[0.0, 0.0, 0.0], [0.15, 0.0, 0.0]], np.float32)
    r = np.full(2, 0.1, np.float32)
    fl = np.ones(2, np.int32)
    v = np.zeros((2, 3), np.float32)
    d = O.particle_contact_deltas(x, v, np.ones(2, np.float32), r, fl, 0.2, DIMS, MU, 0.0, 0.1, 1e-3, 1.0)
    np.testing.assert_allclose(d, [[-0.025, 0, 0], [0.025, 0, 0]], rtol=1e-6)
    # a kinematic partner (inverse mass 0) takes no correction; the other takes all of it
    d = O.particle_contact_deltas(x, v, np.array([1.0, 0.0], np.float32), r, fl, 0.2, DIMS, MU, 0.0, 0.1, 1e-3, 0.5)
    np.testing.assert_allclose(d, [[-0.025, 0, 0], [0.0, 0, 0]], rtol=1e-6)
    # both kinematic: nothing; deltas accumulate onto the initial values
    init = np.ones((2, 3), np.float32)
    d = O.particle_contact_deltas(x, v, np.zeros(2, np.float32), r, fl, 0.2, DIMS, MU, 0.0, 0.1, 1e-3, 1.0,
                                  deltas_init=init)
    np.testing.assert_array_equal(d, init)
    # sliding: friction correction against the tangential motion, at most mu |lambda_n|
    v = np.array([[0.0, 10.0, 0.0], [0.0, 0.0, 0.0]], np.float32)
    d = O.particle_contact_deltas(x, v, np.ones(2, np.float32), r, fl, 0.2, DIMS, MU, 0.0, 0.1, 1e-3, 1.0)
    # lambda_f = max(mu * (-0.05), -|vt| dt) = max(-0.025, -0.01) = -0.01 along +y, halved by denom 2
    np.testing.assert_allclose(d[0], [-0.025, -0.005, 0.0], rtol=1e-5)


def _brute_forces(x, v, r, flags, cohesion, rmax):
    x, v, r = (np.asarray(a, np.float64) for a in (x, v, r))
    n = len(x)
    f = np.zeros((n, 3))
    for i in range(n):
        if not flags[i] & 1:
            continue
        for j in range(n):
            if j == i or not flags[j] & 1:
                continue
            nv = x[i] - x[j]
            d = np.linalg.norm(nv)
            if d > r[i] + rmax + cohesion + 1e-6:
                continue
            err = d - r[i] - r[j]
            if err <= cohesion:
                nv = nv / d
                vr = v[i] - v[j]
                vn = nv @ vr
                fn = err * KE + min(vn, 0.0) * KD
                vt = vr - nv * vn
                vs = np.linalg.norm(vt)
                if vs > 0:
                    vt = vt / vs
                ft = min(vs * KF, MU * abs(fn))
                f[i] += -nv * fn - vt * ft
    return f


def test_oracle_matches_brute_force(oracle_mod):
    rng = np.random.default_rng(3)
    n = 400
    x = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    v = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    r = rng.uniform(0.03, 0.06, n).astype(np.float32)
    flags = (rng.uniform(size=n) > 0.05).astype(np.int32)
    cohesion = 0.01
    f = forces(oracle_mod, x, v, r, flags=flags, cohesion=cohesion)
    ref = _brute_forces(x, v, r, flags, cohesion, float(r.max()))
    act = flags != 0
    scale = np.abs(ref[act]).max()
    np.testing.assert_allclose(f[act], ref[act], rtol=0, atol=1e-5 * scale)
    assert np.count_nonzero(np.abs(ref[act]).sum(axis=1)) > n // 4  # the scene has contacts
