"""Particle-particle contact on the GPU (nsph_particle_contact_forces /
nsph_particle_contact_deltas and the Newton-shaped wrappers) against the fp32
restatement of the reference's kernels (oracle/contact.c): bit for bit, on a
random cloud with mixed radii, velocities, inactive and kinematic particles
and cohesion."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
DIMS = (128, 128, 128)


def cloud(n=20000, seed=5):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    v = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    r = rng.uniform(0.004, 0.012, n).astype(np.float32)
    flags = (rng.uniform(size=n) > 0.03).astype(np.int32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32)
    w[rng.choice(n, n // 50, replace=False)] = 0.0
    return x, v, r, flags, w


def built_grid(x, grid_radius):
    from newton_sph_dev_b200 import HashGrid

    g = HashGrid(*DIMS, device=DEV)
    g.build(torch.from_numpy(x).to(DEV), grid_radius)
    return g


def test_contact_forces_bit_exact(oracle_mod):
    from newton_sph_dev_b200 import _lib

    x, v, r, flags, _ = cloud()
    n = len(x)
    cohesion = 0.002
    rmax = float(r.max())
    gr = float(np.float32(2 * rmax + cohesion))
    g = built_grid(x, gr)
    T = lambda a: torch.from_numpy(a).to(DEV)
    f = torch.full((n, 3), 7.0, device=DEV)
    p = _lib.NsphContactParams(1000.0, 100.0, 100.0, 0.5, cohesion, rmax)
    L = _lib.load()
    xt, vt, rt, ft = T(x), T(v), T(r), T(flags)
    st = L.nsph_particle_contact_forces(g.id, ctypes.byref(p), n, xt.data_ptr(), vt.data_ptr(), rt.data_ptr(),
                                        ft.data_ptr(), f.data_ptr(), _lib.stream_handle(torch.device(DEV)))
    assert st == 0
    torch.cuda.synchronize()
    ref = oracle_mod.particle_contact_forces(x, v, r, flags, gr, DIMS, 1000.0, 100.0, 100.0, 0.5, cohesion, rmax,
                                             f_init=np.full((n, 3), 7.0, np.float32))
    got = f.cpu().numpy()
    np.testing.assert_array_equal(got, ref)
    assert np.count_nonzero(np.abs(got[flags != 0]).sum(axis=1)) > n // 10  # the cloud has contacts


def test_contact_deltas_bit_exact(oracle_mod):
    from newton_sph_dev_b200 import _lib

    x, v, r, flags, w = cloud(seed=6)
    n = len(x)
    cohesion, dt, relax = 0.001, 1e-3, 0.8
    rmax = float(r.max())
    gr = float(np.float32(2 * rmax + cohesion))
    g = built_grid(x, gr)
    init = np.random.default_rng(1).normal(0, 1e-3, (n, 3)).astype(np.float32)
    T = lambda a: torch.from_numpy(a).to(DEV)
    d = T(init.copy())
    L = _lib.load()
    xt, vt, wt, rt, ft = T(x), T(v), T(w), T(r), T(flags)  # kept alive across the launch
    st = L.nsph_particle_contact_deltas(g.id, n, xt.data_ptr(), vt.data_ptr(), wt.data_ptr(), rt.data_ptr(),
                                        ft.data_ptr(), 0.5, cohesion, rmax, dt, relax, d.data_ptr(),
                                        _lib.stream_handle(torch.device(DEV)))
    assert st == 0
    torch.cuda.synchronize()
    ref = oracle_mod.particle_contact_deltas(x, v, w, r, flags, gr, DIMS, 0.5, cohesion, rmax, dt, relax,
                                             deltas_init=init)
    np.testing.assert_array_equal(d.cpu().numpy(), ref)
    assert not np.array_equal(ref, init)


def test_newton_shaped_wrappers(oracle_mod):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.contacts import eval_particle_contact_forces, solve_particle_particle_contacts

    x, v, r, flags, _ = cloud(n=5000, seed=7)
    b = nsph.ModelBuilder()
    b.add_particles(pos=x.tolist(), vel=v.tolist(), mass=[1.0] * len(x), radius=r.tolist())
    model = b.finalize(DEV)
    model.particle_cohesion = 0.001
    state = model.state()
    f = torch.zeros_like(state.particle_q)
    # before the grid is built on these particles: nothing is written (the reference's kernel returns early)
    eval_particle_contact_forces(model, state, f)
    assert torch.count_nonzero(f) == 0
    gr = 2.0 * model.particle_max_radius + model.particle_cohesion
    model.particle_grid.build(state.particle_q, gr)
    eval_particle_contact_forces(model, state, f)
    d = torch.zeros_like(f)
    solve_particle_particle_contacts(model, state.particle_q, state.particle_qd, d, 1e-3, 0.5)
    torch.cuda.synchronize()
    m = model
    ref_f = oracle_mod.particle_contact_forces(x, v, m.particle_radius.cpu().numpy(), m.particle_flags.cpu().numpy(),
                                               float(np.float32(gr)), DIMS, m.particle_ke, m.particle_kd,
                                               m.particle_kf, m.particle_mu, m.particle_cohesion,
                                               m.particle_max_radius)
    np.testing.assert_array_equal(f.cpu().numpy(), ref_f)
    ref_d = oracle_mod.particle_contact_deltas(x, v, m.particle_inv_mass.cpu().numpy(), m.particle_radius.cpu().numpy(),
                                               m.particle_flags.cpu().numpy(), float(np.float32(gr)), DIMS,
                                               m.particle_mu, m.particle_cohesion, m.particle_max_radius, 1e-3, 0.5)
    np.testing.assert_array_equal(d.cpu().numpy(), ref_d)


def test_contact_argument_checks():
    from newton_sph_dev_b200 import HashGrid, _lib

    L = _lib.load()
    g = HashGrid(*DIMS, device=DEV)
    p = _lib.NsphContactParams(1.0, 1.0, 1.0, 0.5, 0.0, 0.1)
    buf = torch.zeros((10, 3), device=DEV)
    fl = torch.ones(10, dtype=torch.int32, device=DEV)
    rr = torch.full((10,), 0.1, device=DEV)
    s = _lib.stream_handle(torch.device(DEV))
    args = (buf.data_ptr(), buf.data_ptr(), rr.data_ptr(), fl.data_ptr(), buf.data_ptr(), s)
    assert L.nsph_particle_contact_forces(g.id, ctypes.byref(p), 10, *args) == _lib.NSPH_ERR_NOT_BUILT
    g.build(torch.rand((10, 3), device=DEV), 0.2)
    assert L.nsph_particle_contact_forces(g.id, ctypes.byref(p), 9, *args) == _lib.NSPH_ERR_INVALID_ARG
    assert L.nsph_particle_contact_forces(g.id, None, 10, *args) == _lib.NSPH_ERR_INVALID_ARG
    assert L.nsph_particle_contact_forces(g.id, ctypes.byref(p), 10, *args) == _lib.NSPH_OK
    torch.cuda.synchronize()
