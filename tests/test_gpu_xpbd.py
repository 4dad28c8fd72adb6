"""Particle contacts with static shapes and the XPBD / semi-implicit particle
steps on the GPU, through the Newton-shaped API -> the C ABI.

Bars:
  - Model.collide (nsph_soft_contacts_create): contact count, particles,
    shapes, points and normals bit-exact against the oracle, in (particle,
    shape) order, over several blocks of particles, for every shape type
    (ground and finite planes, sphere, box, capsule, cylinder, cone,
    ellipsoid);
  - the contact kernels (forces, XPBD deltas, restitution) and
    apply_particle_deltas bit-exact against the oracle on those contacts;
  - SolverXPBD.step (iterations, particle-particle and particle-shape
    corrections, the reference's buffer ping-pong, restitution) and
    SolverSemiImplicit.step bit-exact against the oracle's restatement over
    several steps;
  - the reference's own tests of the XPBD particle path
    (newton/tests/test_solver_xpbd.py:20-146, 149-225, 228-297).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _scene(n=3000, seed=3, up_axis="Z", restitution=0.5):
    import newton_sph_dev_b200 as nsph

    rng = np.random.default_rng(seed)
    b = nsph.ModelBuilder(up_axis=up_axis)
    pos = rng.random((n, 3)) * np.array([2.0, 2.0, 1.0]) + np.array([-1.0, -1.0, -0.05])
    vel = rng.normal(0, 1.0, (n, 3))
    mass = rng.random(n) + 0.5
    mass[rng.choice(n, n // 50, replace=False)] = 0.0  # kinematic
    flags = (rng.random(n) > 0.03).astype(np.int32)  # a few inactive
    radius = rng.random(n) * 0.02 + 0.02
    b.add_particles(pos=pos, vel=vel, mass=mass, radius=radius, flags=flags)
    cfg = nsph.ModelBuilder.ShapeConfig(ke=3000.0, kd=50.0, kf=500.0, mu=0.7)
    b.add_ground_plane(cfg=cfg)
    b.add_shape_sphere(-1, xform=((0.3, 0.2, 0.4), (0.0, 0.0, 0.0, 1.0)), radius=0.3, cfg=cfg)
    b.add_shape_box(-1, xform=((-0.5, -0.4, 0.3), (0.0, 0.0, 0.38268343, 0.92387953)), hx=0.3, hy=0.2, hz=0.25)
    b.add_shape_plane(plane=(1.0, 0.0, 0.0, 0.9), width=1.0, length=3.0)  # finite, facing +x at x = -0.9
    # the round shapes, each tilted off its local +Z axis
    b.add_shape_capsule(-1, xform=((0.55, -0.5, 0.45), (0.25881905, 0.0, 0.0, 0.96592583)), radius=0.15,
                        half_height=0.2, cfg=cfg)
    b.add_shape_cylinder(-1, xform=((-0.4, 0.55, 0.4), (0.0, 0.38268343, 0.0, 0.92387953)), radius=0.2,
                         half_height=0.15)
    b.add_shape_cone(-1, xform=((0.65, 0.6, 0.3), (0.0, 0.0, 0.0, 1.0)), radius=0.25, half_height=0.2, cfg=cfg)
    b.add_shape_ellipsoid(-1, xform=((0.0, -0.15, 0.65), (0.18301270, 0.18301270, 0.0, 0.96592583)), rx=0.3,
                          ry=0.15, rz=0.1)
    m = b.finalize(DEV)
    m.soft_contact_restitution = restitution
    m.particle_mu = 0.4
    m.particle_cohesion = 0.005
    return m


def _model_dict(m):
    return dict(inv_mass=m.particle_inv_mass.cpu().numpy(), radius=m.particle_radius.cpu().numpy(),
                flags=m.particle_flags.cpu().numpy(), world=m.particle_world.cpu().numpy(),
                gravity=m.gravity.cpu().numpy(), v_max=m.particle_max_velocity, particle_mu=m.particle_mu,
                particle_cohesion=m.particle_cohesion, max_radius=m.particle_max_radius,
                shapes=[dict(type=s["type"], flags=s["flags"], world=s["world"], pos=s["pos"], rot=s["rot"],
                             scale=s["scale"], ke=s["ke"], kd=s["kd"], kf=s["kf"], mu=s["mu"]) for s in m._shapes],
                soft=(m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_kf, m.soft_contact_mu, m.particle_adhesion,
                      m.soft_contact_restitution))


def _contacts_host(c):
    n = int(min(c.soft_contact_max, int(c.soft_contact_count.item())))
    return dict(count=c.soft_contact_count.cpu().numpy(), n=n, particle=c.soft_contact_particle.cpu().numpy(),
                shape=c.soft_contact_shape.cpu().numpy(), body_pos=c.soft_contact_body_pos.cpu().numpy(),
                body_vel=c.soft_contact_body_vel.cpu().numpy(), normal=c.soft_contact_normal.cpu().numpy())


def test_collide_matches_oracle(oracle_mod):
    m = _scene(n=50_000)
    s = m.state()
    c = m.collide(s)
    torch.cuda.synchronize()
    md = _model_dict(m)
    ref = oracle_mod.soft_contacts_create(md["shapes"], s.particle_q.cpu().numpy(), md["radius"], md["flags"],
                                          world=md["world"], margin=0.01)
    got = _contacts_host(c)
    assert got["count"][0] == ref["count"][0] > 1000
    assert set(got["shape"][:got["n"]].tolist()) == set(range(len(md["shapes"]))), "every shape makes contacts"
    k = ref["n"]
    for key in ("particle", "shape", "body_pos", "body_vel", "normal"):
        np.testing.assert_array_equal(got[key][:k], ref[key][:k], err_msg=key)
    # a capacity below the count keeps the first contacts and reports the total
    small = m.contacts(soft_contact_max=100)
    m.collide(s, small)
    torch.cuda.synchronize()
    g2 = _contacts_host(small)
    assert g2["count"][0] == ref["count"][0]
    np.testing.assert_array_equal(g2["particle"][:100], ref["particle"][:100])


def test_shape_contact_kernels_match_oracle(oracle_mod):
    from newton_sph_dev_b200 import contacts as pc

    m = _scene(n=20_000, seed=5)
    s = m.state()
    c = m.collide(s)
    md = _model_dict(m)
    x, v = s.particle_q.cpu().numpy(), s.particle_qd.cpu().numpy()
    ch = _contacts_host(c)
    # semi-implicit forces, subtracted from existing forces
    f0 = torch.randn_like(s.particle_q)
    f = f0.clone()
    pc.eval_particle_body_contact_forces(m, s, c, f)
    prm = oracle_mod.soft_contact_params(*md["soft"], 0.0, 0.0)
    ref = oracle_mod.shape_contact_forces(md["shapes"], ch, prm, x, v, md["radius"], md["flags"], f0.cpu().numpy())
    np.testing.assert_array_equal(f.cpu().numpy(), ref)
    # XPBD corrections
    d0 = torch.randn_like(s.particle_q) * 1e-3
    d = d0.clone()
    pc.solve_particle_shape_contacts(m, s.particle_q, s.particle_qd, c, d, 1e-3, 0.8)
    prm = oracle_mod.soft_contact_params(*md["soft"], 0.8, 1e-3)
    ref = oracle_mod.shape_contact_deltas(md["shapes"], ch, prm, x, v, md["inv_mass"], md["radius"], md["flags"],
                                          d0.cpu().numpy())
    np.testing.assert_array_equal(d.cpu().numpy(), ref)
    # restitution (v_new aliasing v_out, as in the solver)
    vn = torch.randn_like(s.particle_qd)
    vref = oracle_mod.shape_restitution(ch, prm, vn.cpu().numpy(), x, v, md["radius"], md["flags"], vn.cpu().numpy())
    pc.apply_particle_shape_restitution(m, c, vn, s.particle_q, s.particle_qd, vn)
    np.testing.assert_array_equal(vn.cpu().numpy(), vref)
    # apply_particle_deltas with the velocity clamp active for some particles
    m.particle_max_velocity = 3.0
    xo = torch.full_like(s.particle_q, -1.0)
    vo = torch.full_like(s.particle_q, -1.0)
    xp = s.particle_q + torch.randn_like(s.particle_q) * 1e-3
    pc.apply_particle_deltas(m, s.particle_q, xp, d, 1e-3, xo, vo)
    xr = np.full_like(x, -1.0)
    vr = np.full_like(x, -1.0)
    oracle_mod.apply_particle_deltas(x, xp.cpu().numpy(), md["flags"], d.cpu().numpy(), 1e-3, 3.0, xr, vr)
    np.testing.assert_array_equal(xo.cpu().numpy(), xr)
    np.testing.assert_array_equal(vo.cpu().numpy(), vr)


@pytest.mark.parametrize("iterations,restitution", [(4, True), (3, False)])
def test_xpbd_step_matches_oracle(oracle_mod, iterations, restitution):
    from newton_sph_dev_b200.solvers import SolverXPBD

    m = _scene(n=4000, seed=7)
    md = _model_dict(m)
    solver = SolverXPBD(m, iterations=iterations, soft_contact_relaxation=0.8, enable_restitution=restitution)
    s0, s1 = m.state(), m.state()
    s0.particle_f.normal_(0, 0.5)
    dt = 2e-3
    h0 = [s0.particle_q.cpu().numpy(), s0.particle_qd.cpu().numpy(), s0.particle_f.cpu().numpy()]
    h1 = [s1.particle_q.cpu().numpy(), s1.particle_qd.cpu().numpy(), s1.particle_f.cpu().numpy()]
    for _ in range(3):
        c = m.collide(s0)
        ch = _contacts_host(c)
        solver.step(s0, s1, m.control(), c, dt)
        torch.cuda.synchronize()
        ref_c = oracle_mod.soft_contacts_create(md["shapes"], h0[0], md["radius"], md["flags"], world=md["world"],
                                                margin=0.01)
        assert ref_c["count"][0] == ch["count"][0]
        xi, vi, xo, vo = oracle_mod.xpbd_particle_step(md, h0[0], h0[1], h0[2], dt, iterations, 0.8, contacts=ref_c,
                                                       enable_restitution=restitution, x_out_init=h1[0],
                                                       v_out_init=h1[1])
        np.testing.assert_array_equal(s1.particle_q.cpu().numpy(), xo)
        np.testing.assert_array_equal(s1.particle_qd.cpu().numpy(), vo)
        np.testing.assert_array_equal(s0.particle_q.cpu().numpy(), xi)
        np.testing.assert_array_equal(s0.particle_qd.cpu().numpy(), vi)
        h0, h1 = [xo, vo, h1[2]], [xi, vi, h0[2]]
        s0, s1 = s1, s0
    assert np.all(np.isfinite(h0[0]))


def test_semi_implicit_step_matches_oracle(oracle_mod):
    from newton_sph_dev_b200.solvers import SolverSemiImplicit

    m = _scene(n=4000, seed=11)
    md = _model_dict(m)
    solver = SolverSemiImplicit(m)
    s0, s1 = m.state(), m.state()
    s0.particle_f.normal_(0, 0.5)
    dt = 1e-4
    grid_r = m.particle_max_radius * 2.0 + m.particle_cohesion
    for _ in range(3):
        x, v, f = s0.particle_q.cpu().numpy(), s0.particle_qd.cpu().numpy(), s0.particle_f.cpu().numpy()
        v_out0 = s1.particle_qd.cpu().numpy()
        m.particle_grid.build(s0.particle_q, grid_r)
        c = m.collide(s0)
        solver.step(s0, s1, None, c, dt)
        torch.cuda.synchronize()
        ch = _contacts_host(c)
        fr = oracle_mod.particle_contact_forces(x, v, md["radius"], md["flags"], grid_r, (128, 128, 128),
                                                m.particle_ke, m.particle_kd, m.particle_kf, m.particle_mu,
                                                m.particle_cohesion, m.particle_max_radius, f_init=f)
        prm = oracle_mod.soft_contact_params(*md["soft"], 0.0, 0.0)
        fr = oracle_mod.shape_contact_forces(md["shapes"], ch, prm, x, v, md["radius"], md["flags"], fr)
        np.testing.assert_array_equal(s0.particle_f.cpu().numpy(), fr)
        xn, vn = np.zeros_like(x), v_out0.copy()
        oracle_mod.integrate_particles(x, v, fr, md["inv_mass"], md["flags"], md["world"], md["gravity"], dt,
                                       m.particle_max_velocity, xn, vn)
        np.testing.assert_array_equal(s1.particle_q.cpu().numpy(), xn)
        np.testing.assert_array_equal(s1.particle_qd.cpu().numpy(), vn)
        s0, s1 = s1, s0


# ---- the reference's own XPBD particle tests (newton/tests/test_solver_xpbd.py)
def _two_particles(v0, v1, mu):
    import newton_sph_dev_b200 as nsph

    b = nsph.ModelBuilder(up_axis="Y")
    sep = 2.0 * 0.5 - 0.1
    b.add_particles(pos=[(0.0, 0.0, 0.0), (sep, 0.0, 0.0)], vel=[v0, v1], mass=[1.0, 1.0], radius=[0.5, 0.5])
    m = b.finalize(DEV)
    m.set_gravity((0.0, 0.0, 0.0))
    m.particle_mu = mu
    m.particle_cohesion = 0.0
    return m


def test_reference_particle_particle_friction_uses_relative_velocity():
    """test_solver_xpbd.py:20-146."""
    from newton_sph_dev_b200.solvers import SolverXPBD

    model = _two_particles((0.0, 0.0, 10.0), (0.0, 0.0, 10.0), 1.0)
    solver = SolverXPBD(model=model, iterations=20)
    state0, state1 = model.state(), model.state()
    contacts = model.contacts()
    state0.particle_f.copy_(torch.tensor([[50.0, 0.0, 0.0], [-50.0, 0.0, 0.0]], device=DEV))
    initial = state0.particle_qd.cpu().numpy().copy()
    for _ in range(60):
        model.collide(state0, contacts)
        solver.step(state0, state1, model.control(), contacts, 1.0 / 60.0)
        state0, state1 = state1, state0
    final = state0.particle_qd.cpu().numpy()
    assert round(initial[0, 2] - initial[1, 2], 5) == 0.0
    assert round(final[0, 2] - final[1, 2], 3) == 0.0
    assert round(final[0, 2] - final[1, 2], 3) == 0.0 and abs(final[0, 2]) > 1.0


def test_reference_particle_particle_friction_with_relative_motion():
    """test_solver_xpbd.py:149-225."""
    from newton_sph_dev_b200.solvers import SolverXPBD

    def run(mu):
        model = _two_particles((0.0, 0.0, 10.0), (0.0, 0.0, 0.0), mu)
        solver = SolverXPBD(model=model, iterations=30)
        state0, state1 = model.state(), model.state()
        contacts = model.contacts()
        model.collide(state0, contacts)
        solver.step(state0, state1, model.control(), contacts, 1.0 / 30.0)
        q1 = state1.particle_q.cpu().numpy()
        return float(abs(q1[0, 2] - q1[1, 2]))

    slip_no_friction = run(0.0)
    slip_with_friction = run(1.0)
    assert slip_no_friction > 0.2
    assert slip_with_friction < slip_no_friction * 0.95


def test_reference_particle_shape_restitution_correct_particle():
    """test_solver_xpbd.py:228-297."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverXPBD

    builder = nsph.ModelBuilder(up_axis="Y")
    builder.add_particle(pos=(0.0, 10.0, 0.0), vel=(0.0, 0.0, 0.0), mass=1.0, radius=0.1)
    builder.add_particle(pos=(0.0, 0.1, 0.0), vel=(0.0, -5.0, 0.0), mass=1.0, radius=0.1)
    builder.add_ground_plane()
    model = builder.finalize(DEV)
    model.set_gravity((0.0, 0.0, 0.0))
    model.soft_contact_restitution = 1.0
    solver = SolverXPBD(model=model, iterations=10, enable_restitution=True)
    state0, state1 = model.state(), model.state()
    contacts = model.contacts()
    model.collide(state0, contacts)
    solver.step(state0, state1, model.control(), contacts, 1.0 / 60.0)
    vel = state1.particle_qd.cpu().numpy()
    assert round(float(vel[0, 1]), 2) == 0.0
    assert float(vel[1, 1]) > 0.0


def test_xpbd_refuses_rigid_models():
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverXPBD

    b = nsph.ModelBuilder()
    with pytest.raises(NotImplementedError):
        b.add_shape_sphere(0, radius=1.0)
    b.add_particle((0, 0, 0), (0, 0, 0), 1.0)
    m = b.finalize(DEV)
    m.body_count = 1
    with pytest.raises(NotImplementedError):
        SolverXPBD(m)
