"""The oracle's particle-shape contacts and XPBD particle step, on the CPU.

Pins oracle/shapes.c (the restatement the GPU kernels are checked against):

  - known answers of the soft-contact generation (create_soft_contacts,
    newton/_src/geometry/kernels.py:1001-1140): sphere, box (outside and
    inside), infinite and finite plane, a plane rotated onto +Y, the margin,
    the COLLIDE_PARTICLES flag and the world filter;
  - known answers of the capsule, cylinder, cone and ellipsoid SDFs
    (sdf_capsule / sdf_cylinder / sdf_cone / sdf_ellipsoid and their
    gradients, newton/_src/geometry/kernels.py:132-565);
  - the signed distances and contact points of random particles against an
    fp64 numpy restatement of the SDFs (capsule, cylinder and cone from
    their exact distances: to a segment, to a rectangle and to a triangle in
    the (radius, z) half plane);
  - known answers of the contact laws (eval_particle_body_contact,
    solve_particle_shape_contacts, apply_particle_shape_restitution) and of
    apply_particle_deltas (newton/_src/solvers/xpbd/kernels.py:777-808);
  - the reference's own behavioural tests of the XPBD particle path
    (newton/tests/test_solver_xpbd.py:20-146, 149-225, 228-297), run on the
    oracle's restatement of SolverXPBD.step.
"""

from __future__ import annotations

import numpy as np
import pytest

PLANE, SPHERE, CAPSULE, ELLIPSOID, CYLINDER, BOX, CONE = 1, 3, 4, 5, 6, 7, 9
COLLIDE = 1 << 2


def _model_dict(model, soft=None):
    m = dict(inv_mass=model.particle_inv_mass.numpy(), radius=model.particle_radius.numpy(),
             flags=model.particle_flags.numpy(), world=model.particle_world.numpy(), gravity=model.gravity.numpy(),
             v_max=model.particle_max_velocity, particle_mu=model.particle_mu,
             particle_cohesion=model.particle_cohesion, max_radius=model.particle_max_radius,
             shapes=[dict(type=s["type"], flags=s["flags"], world=s["world"], pos=s["pos"], rot=s["rot"],
                          scale=s["scale"], ke=s["ke"], kd=s["kd"], kf=s["kf"], mu=s["mu"]) for s in model._shapes])
    m["soft"] = soft if soft is not None else (model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_kf,
                                               model.soft_contact_mu, model.particle_adhesion,
                                               model.soft_contact_restitution)
    return m


def test_soft_contact_known_answers(oracle_mod):
    O = oracle_mod
    r = 0.1
    shapes = [dict(type=SPHERE, pos=(0, 0, 0), scale=(1.0, 0, 0)),
              dict(type=PLANE, scale=(0, 0, 0)),
              dict(type=BOX, pos=(3, 0, 0), scale=(0.5, 0.5, 0.5)),
              dict(type=PLANE, pos=(10, 0, 0), scale=(2.0, 2.0, 0)),  # finite plane, 1 x 1 half extents
              dict(type=SPHERE, pos=(0, 0, 0), scale=(1.0, 0, 0), flags=0),  # no particle collision
              dict(type=SPHERE, pos=(0, 0, 0), scale=(1.0, 0, 0), world=5)]  # another world
    x = np.array([[0, 0, 1.05],    # sphere (d = 0.05 < 0.11), plane too far (z = 1.05)
                  [0, 0, 0.05],    # inside the sphere and on the plane
                  [3.6, 0, 0],     # box +x face and the plane
                  [3.2, 0, 0.3],   # inside the box: nearest face +z; plane z = 0.3 too far
                  [10.5, 0.5, 0.05],  # finite plane and the infinite one
                  [50, 50, 50]], np.float32)
    c = O.soft_contacts_create(shapes, x, np.full(len(x), r, np.float32), np.ones(len(x), np.int32),
                               world=np.zeros(len(x), np.int32), margin=0.01)
    got = list(zip(c["particle"][:c["n"]].tolist(), c["shape"][:c["n"]].tolist()))
    assert got == [(0, 0), (1, 0), (1, 1), (2, 1), (2, 2), (3, 2), (4, 1), (4, 3)]
    bp, nn = c["body_pos"][:c["n"]], c["normal"][:c["n"]]
    np.testing.assert_allclose(bp[0], [0, 0, 1], atol=1e-7)
    np.testing.assert_allclose(nn[0], [0, 0, 1])
    np.testing.assert_allclose(bp[1], [0, 0, 1], atol=1e-7)  # x - n d with d = -0.95
    np.testing.assert_allclose(bp[4], [3.5, 0, 0], atol=1e-7)
    np.testing.assert_allclose(nn[4], [1, 0, 0])
    np.testing.assert_allclose(bp[5], [3.2, 0, 0.5], atol=1e-7)  # inside: pushed out through +z
    np.testing.assert_allclose(nn[5], [0, 0, 1])
    # finite plane: Chebyshev distance max(max(|x|-w, |y|-l), |z|) = 0.05
    np.testing.assert_allclose(bp[7], [10.5, 0.5, 0.0], atol=1e-6)
    # max clamps the writes, not the count
    c2 = O.soft_contacts_create(shapes, x, np.full(len(x), r, np.float32), np.ones(len(x), np.int32),
                                world=np.zeros(len(x), np.int32), margin=0.01, max_contacts=3)
    assert c2["count"][0] == 8 and c2["n"] == 3
    # global particles (world -1) meet the shapes of every world
    c4 = O.soft_contacts_create(shapes, x, np.full(len(x), r, np.float32), np.ones(len(x), np.int32), margin=0.01)
    assert c4["count"][0] == 10
    # inactive particles make no contacts
    fl = np.ones(len(x), np.int32)
    fl[1] = 0
    c3 = O.soft_contacts_create(shapes, x, np.full(len(x), r, np.float32), fl, margin=0.01)
    assert 1 not in c3["particle"][:c3["n"]].tolist()


def test_ground_plane_up_y(oracle_mod):
    """add_ground_plane with up_axis Y: the plane's local +Z maps to world +Y."""
    import newton_sph_dev_b200 as nsph

    b = nsph.ModelBuilder(up_axis="Y")
    b.add_particle((0.0, 0.05, 0.0), (0.0, 0.0, 0.0), 1.0, radius=0.1)
    b.add_particle((0.0, 5.0, 0.0), (0.0, 0.0, 0.0), 1.0, radius=0.1)
    b.add_ground_plane()
    m = b.finalize("cpu")
    md = _model_dict(m)
    c = oracle_mod.soft_contacts_create(md["shapes"], m.particle_q.numpy(), md["radius"], md["flags"], margin=0.01)
    assert c["n"] == 1 and c["particle"][0] == 0
    np.testing.assert_allclose(c["normal"][0], [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(c["body_pos"][0], [0, 0, 0], atol=1e-6)


def _sdf64(s, p):
    """fp64 signed distance and contact point of a static shape (axis-aligned)."""
    q = p - np.asarray(s["pos"], np.float64)
    if s["type"] == SPHERE:
        ln = np.linalg.norm(q)
        n = q / ln
        d = ln - s["scale"][0]
    elif s["type"] == BOX:
        h = np.asarray(s["scale"], np.float64)
        qa = np.abs(q) - h
        d = np.linalg.norm(np.maximum(qa, 0)) + min(max(qa), 0.0)
        if np.any(qa > 0):
            c = np.clip(q, -h, h)
            n = (q - c) / np.linalg.norm(q - c)
        else:
            k = int(np.argmax(qa))
            n = np.zeros(3)
            n[k] = np.sign(q[k]) if q[k] != 0 else 1.0
    else:
        d = q[2]
        n = np.array([0.0, 0.0, 1.0])
    return d, np.asarray(s["pos"]) + q - n * d, n


def test_round_shape_known_answers(oracle_mod):
    """Capsule, cylinder, cone and ellipsoid contacts at points whose
    distance, contact point and normal are known in closed form."""
    O = oracle_mod
    shapes = [dict(type=CAPSULE, pos=(0, 0, 0), scale=(0.5, 1.0, 0)),
              dict(type=CYLINDER, pos=(5, 0, 0), scale=(0.5, 1.0, 0)),
              dict(type=CONE, pos=(10, 0, 0), scale=(0.5, 0.5, 0)),
              dict(type=ELLIPSOID, pos=(15, 0, 0), scale=(1.0, 0.5, 0.5))]
    s5 = 1.0 / np.sqrt(5.0)
    x = np.array([[0.7, 0, 0.2],      # capsule side: d 0.2
                  [0, 0, 1.6],        # capsule top cap: d 0.1
                  [0, 0, -1.55],      # capsule bottom cap: d 0.05
                  [0, 0, 0.3],        # on the capsule axis: the fallback normal +z, d -0.5
                  [5.6, 0, 0],        # cylinder side: d 0.1
                  [5, 0, 1.05],       # cylinder top: d 0.05
                  [5.6, 0, 1.1],      # cylinder rim: d 0.1 sqrt 2 along (1, 0, 1) / sqrt 2
                  [5.2, 0, 0.9],      # inside the cylinder, nearest the top: d -0.1
                  [10, 0, 0.6],       # above the cone's apex: d 0.1
                  [10, 0, -0.55],     # below the cone's base: d 0.05
                  [10 + 0.25 + 0.1 * 2 * s5, 0, 0.1 * s5],  # off the cone's side by 0.1 along (2, 0, 1) / sqrt 5
                  [17, 0, 0],         # ellipsoid: 1 beyond the x semi-axis
                  [15, 0.7, 0]],      # ellipsoid: 0.2 beyond the y semi-axis
                 np.float32)
    r = np.full(len(x), 0.1, np.float32)
    c = O.soft_contacts_create(shapes, x, r, np.ones(len(x), np.int32), margin=0.85)
    got = list(zip(c["particle"][:c["n"]].tolist(), c["shape"][:c["n"]].tolist()))
    assert got == [(0, 0), (1, 0), (2, 0), (3, 0), (4, 1), (5, 1), (6, 1), (7, 1), (8, 2), (9, 2), (10, 2),
                   (12, 3)]  # particle 11 is 1 from the ellipsoid, beyond margin + radius = 0.95
    bp, nn = c["body_pos"][:c["n"]], c["normal"][:c["n"]]
    want_bp = [[0.5, 0, 0.2], [0, 0, 1.5], [0, 0, -1.5], [0, 0, 0.8], [5.5, 0, 0], [5, 0, 1], [5.5, 0, 1.0],
               [5.2, 0, 1.0], [10, 0, 0.5], [10, 0, -0.5], [10.25, 0, 0], [15, 0.5, 0]]
    want_n = [[1, 0, 0], [0, 0, 1], [0, 0, -1], [0, 0, 1], [1, 0, 0], [0, 0, 1], [np.sqrt(0.5), 0, np.sqrt(0.5)],
              [0, 0, 1], [0, 0, 1], [0, 0, -1], [2 * s5, 0, s5], [0, 1, 0]]
    np.testing.assert_allclose(bp, want_bp, atol=2e-6)
    np.testing.assert_allclose(nn, want_n, atol=2e-6)
    c3 = O.soft_contacts_create(shapes[3:], x[11:12], r[11:12], np.ones(1, np.int32), margin=0.95)
    assert c3["n"] == 1
    np.testing.assert_allclose(c3["body_pos"][0], [16, 0, 0], atol=2e-6)


def _tri_dist2d(p, a, b):
    """Distance from 2-D point p to the segment a-b."""
    ab, ap = b - a, p - a
    t = np.clip(np.dot(ap, ab) / np.dot(ab, ab), 0.0, 1.0)
    return np.linalg.norm(ap - t * ab)


def _round_sdf64(s, q):
    """fp64 signed distance and outward normal of an axis-aligned capsule,
    cylinder, cone or ellipsoid at local point q. Capsule, cylinder and cone
    from their exact distances; the cone's normal and the ellipsoid (whose
    SDF is the reference's approximation) restate the reference's formulas."""
    r, hh = float(s["scale"][0]), float(s["scale"][1])
    rho = np.hypot(q[0], q[1])
    radial = np.array([q[0] / rho, q[1] / rho, 0.0]) if rho > 1e-8 else np.array([0.0, 0.0, 1.0])
    axial = np.array([0.0, 0.0, 1.0 if q[2] >= 0 else -1.0])
    if s["type"] == CAPSULE:
        v = q - np.array([0.0, 0.0, np.clip(q[2], -hh, hh)])
        ln = np.linalg.norm(v)
        return ln - r, v / ln
    if s["type"] == CYLINDER:
        dx, dy = rho - r, abs(q[2]) - hh
        d = min(max(dx, dy), 0.0) + np.hypot(max(dx, 0.0), max(dy, 0.0))
        if dx > 0 and dy > 0:
            g = radial * dx + axial * dy
            return d, g / np.linalg.norm(g)
        return d, radial if dx > dy else axial
    if s["type"] == CONE:
        p2 = np.array([rho, q[2]])
        base = (np.array([0.0, -hh]), np.array([r, -hh]))
        side = (np.array([r, -hh]), np.array([0.0, hh]))
        dist = min(_tri_dist2d(p2, *base), _tri_dist2d(p2, *side))
        inside = -hh <= q[2] <= hh and rho <= r * (hh - q[2]) / (2 * hh)
        d = -dist if inside else dist
        dx, dy = rho - r * (hh - q[2]) / (2 * hh), abs(q[2]) - hh
        if dx > dy:
            g = radial + np.array([0.0, 0.0, r / (2 * hh)])
            return d, g / np.linalg.norm(g)
        return d, axial
    rr = np.abs(np.asarray(s["scale"], np.float64))
    q0, q1 = q / rr, q / rr**2
    k0, k1 = np.linalg.norm(q0), np.linalg.norm(q1)
    g = q1 * (k0 / k1)
    return k0 * (k0 - 1.0) / k1, g / np.linalg.norm(g)


def test_round_shapes_against_fp64(oracle_mod):
    rng = np.random.default_rng(7)
    shapes = [dict(type=CAPSULE, pos=(0.1, 0.2, -0.1), scale=(0.3, 0.5, 0)),
              dict(type=CYLINDER, pos=(-0.8, 0.4, 0.2), scale=(0.35, 0.25, 0)),
              dict(type=CONE, pos=(0.7, -0.6, 0.1), scale=(0.4, 0.45, 0)),
              dict(type=ELLIPSOID, pos=(-0.5, -0.7, -0.4), scale=(0.5, 0.3, 0.2))]
    x = (rng.random((6000, 3)) * 3 - 1.5).astype(np.float32)
    r = (rng.random(6000) * 0.05 + 0.01).astype(np.float32)
    margin = 0.05
    c = oracle_mod.soft_contacts_create(shapes, x, r, np.ones(len(x), np.int32), margin=margin)
    want, near = set(), set()
    for i in range(len(x)):
        for k, s in enumerate(shapes):
            d, _ = _round_sdf64(s, x[i].astype(np.float64) - np.asarray(s["pos"], np.float64))
            if d < margin + r[i] - 1e-5:
                want.add((i, k))
            elif d < margin + r[i] + 1e-5:
                near.add((i, k))  # within rounding of the threshold: either way
    got = set(zip(c["particle"][:c["n"]].tolist(), c["shape"][:c["n"]].tolist()))
    assert want <= got <= want | near
    assert all(any(k == t for _, k in want) for t in range(4)), "every shape makes contacts"
    for t in range(c["n"]):
        i, k = int(c["particle"][t]), int(c["shape"][t])
        pos = np.asarray(shapes[k]["pos"], np.float64)
        q = x[i].astype(np.float64) - pos
        d, n = _round_sdf64(shapes[k], q)
        np.testing.assert_allclose(c["normal"][t], n, atol=5e-6, err_msg=f"shape {k}")
        np.testing.assert_allclose(c["body_pos"][t], pos + q - n * d, atol=5e-6, err_msg=f"shape {k}")


def test_site_shapes_make_no_contacts(oracle_mod):
    import newton_sph_dev_b200 as nsph

    b = nsph.ModelBuilder()
    b.add_particle((0.0, 0.0, 0.05), (0.0, 0.0, 0.0), 1.0, radius=0.1)
    b.add_shape_capsule(-1, radius=0.2, half_height=0.1, as_site=True)
    b.add_shape_cone(-1, radius=0.2, half_height=0.1)
    m = b.finalize("cpu")
    md = _model_dict(m)
    assert [s["type"] for s in md["shapes"]] == [CAPSULE, CONE]
    assert [s["scale"] for s in md["shapes"]] == [(0.2, 0.1, 0.0), (0.2, 0.1, 0.0)]
    c = oracle_mod.soft_contacts_create(md["shapes"], m.particle_q.numpy(), md["radius"], md["flags"], margin=0.01)
    assert c["n"] == 1 and c["shape"][0] == 1


def test_soft_contacts_against_fp64(oracle_mod):
    rng = np.random.default_rng(4)
    shapes = [dict(type=SPHERE, pos=(0.2, -0.1, 0.3), scale=(0.7, 0, 0)),
              dict(type=BOX, pos=(-1.0, 0.5, 0.0), scale=(0.4, 0.3, 0.6)),
              dict(type=PLANE, pos=(0, 0, -1.0), scale=(0, 0, 0))]
    x = (rng.random((4000, 3)) * 4 - 2).astype(np.float32)
    r = (rng.random(4000) * 0.05 + 0.01).astype(np.float32)
    margin = 0.05
    c = oracle_mod.soft_contacts_create(shapes, x, r, np.ones(len(x), np.int32), margin=margin)
    want = []
    for i in range(len(x)):
        for k, s in enumerate(shapes):
            d, _, _ = _sdf64(s, x[i].astype(np.float64))
            if d < margin + r[i] - 1e-5:
                want.append((i, k))
            elif d < margin + r[i] + 1e-5:
                want.append(None)  # within rounding of the threshold: either way
    got = set(zip(c["particle"][:c["n"]].tolist(), c["shape"][:c["n"]].tolist()))
    assert {w for w in want if w is not None} <= got
    assert len(got) <= len(want)
    for t in range(c["n"]):
        i, k = int(c["particle"][t]), int(c["shape"][t])
        _, cp, n = _sdf64(shapes[k], x[i].astype(np.float64))
        np.testing.assert_allclose(c["body_pos"][t], cp, atol=2e-6)
        np.testing.assert_allclose(c["normal"][t], n, atol=2e-6)


def test_contact_laws_known_answers(oracle_mod):
    O = oracle_mod
    shapes = [dict(type=PLANE, scale=(0, 0, 0), ke=2000.0, kd=20.0, kf=100.0, mu=0.8)]
    # one particle 0.02 into the ground (radius 0.1 at z = 0.08), moving down and sideways
    x = np.array([[0.0, 0.0, 0.08]], np.float32)
    v = np.array([[1.0, 0.0, -2.0]], np.float32)
    r = np.array([0.1], np.float32)
    fl = np.ones(1, np.int32)
    c = O.soft_contacts_create(shapes, x, r, fl, margin=0.01)
    assert c["n"] == 1
    prm = O.soft_contact_params(1000.0, 10.0, 1000.0, 0.5, 0.0, 0.5, 0.9, 0.01)
    f = O.shape_contact_forces(shapes, c, prm, x, v, r, fl, np.zeros((1, 3), np.float32))
    ke, kd, kf, mu = 1500.0, 15.0, 550.0, 0.65
    cc = -0.02
    fn = cc * ke  # along n = +z
    fd = -2.0 * kd
    ft = min(kf * 1.0, abs(mu * cc * ke))
    np.testing.assert_allclose(f[0], [-ft, 0.0, -(fn + fd)], rtol=1e-5)
    # XPBD: push out along n by relaxation * 0.02 (w = 1), friction capped by mu*c
    w = np.ones(1, np.float32)
    d = O.shape_contact_deltas(shapes, c, prm, x, v, w, r, fl, np.zeros((1, 3), np.float32))
    lam_f = max(mu * cc, -1.0 * 0.01)
    np.testing.assert_allclose(d[0], [lam_f * 0.9, 0.0, 0.02 * 0.9], rtol=1e-5)
    # kinematic particle (w = 0): no correction
    d0 = O.shape_contact_deltas(shapes, c, prm, x, v, np.zeros(1, np.float32), r, fl, np.zeros((1, 3), np.float32))
    assert np.all(d0 == 0)
    # restitution: approaching at -2, now moving at -0.5 -> v gains n (0.5 + 0.5 * 2)
    vo = O.shape_restitution(c, prm, np.array([[1.0, 0.0, -0.5]], np.float32), x, v, r, fl,
                             np.array([[1.0, 0.0, -0.5]], np.float32))
    np.testing.assert_allclose(vo[0], [1.0, 0.0, 1.0], rtol=1e-6)
    # receding contact: no restitution
    vo2 = O.shape_restitution(c, prm, v, x, np.array([[0.0, 0.0, 1.0]], np.float32), r, fl, v.copy())
    np.testing.assert_array_equal(vo2, v)


def test_apply_particle_deltas(oracle_mod):
    x0 = np.array([[0, 0, 0], [1, 1, 1], [2, 2, 2]], np.float32)
    xp = np.array([[0.1, 0, 0], [1, 1, 1.5], [2, 2, 2]], np.float32)
    d = np.array([[0.1, 0, 0], [0, 0, 0], [9, 9, 9]], np.float32)
    fl = np.array([1, 1, 0], np.int32)
    xo = np.full((3, 3), -1, np.float32)
    vo = np.full((3, 3), -1, np.float32)
    oracle_mod.apply_particle_deltas(x0, xp, fl, d, 0.1, 3.0, xo, vo)
    np.testing.assert_allclose(xo[0], [0.2, 0, 0], rtol=1e-6)
    np.testing.assert_allclose(vo[0], [2.0, 0, 0], rtol=1e-6)
    np.testing.assert_allclose(vo[1], [0, 0, 3.0], rtol=1e-6)  # 5 m/s clamped to 3
    assert np.all(xo[2] == -1) and np.all(vo[2] == -1)  # inactive: untouched


# ---- the reference's XPBD particle tests (newton/tests/test_solver_xpbd.py), on the oracle
def _two_particles(v0, v1, mu):
    import newton_sph_dev_b200 as nsph

    b = nsph.ModelBuilder(up_axis="Y")
    sep = 2.0 * 0.5 - 0.1
    b.add_particles(pos=[(0.0, 0.0, 0.0), (sep, 0.0, 0.0)], vel=[v0, v1], mass=[1.0, 1.0], radius=[0.5, 0.5])
    m = b.finalize("cpu")
    m.set_gravity((0.0, 0.0, 0.0))
    m.particle_mu = mu
    m.particle_cohesion = 0.0
    return m


def test_reference_friction_uses_relative_velocity(oracle_mod):
    """test_solver_xpbd.py:20-146: equal tangential velocities stay equal."""
    m = _two_particles((0.0, 0.0, 10.0), (0.0, 0.0, 10.0), 1.0)
    md = _model_dict(m)
    s0 = [m.particle_q.numpy().copy(), m.particle_qd.numpy().copy(), np.array([[50, 0, 0], [-50, 0, 0]], np.float32)]
    s1 = [m.particle_q.numpy().copy(), m.particle_qd.numpy().copy(), np.zeros((2, 3), np.float32)]
    for _ in range(60):
        # two particles: the grid's dims do not change their candidates, so a
        # small grid keeps the 1200 oracle grid builds quick
        xi, vi, xo, vo = oracle_mod.xpbd_particle_step(md, s0[0], s0[1], s0[2], 1.0 / 60.0, 20, 0.9, dims=(8, 8, 8))
        s0[0], s0[1] = xi, vi  # the step writes into its input state's buffers too
        s1[0], s1[1] = xo, vo
        s0, s1 = s1, s0
    vf = s0[1]
    # the reference asserts equality to 3 places and that both keep moving together
    assert abs(vf[0, 2] - vf[1, 2]) < 5e-4 and abs(vf[0, 2]) > 1.0


def test_reference_friction_reduces_slip(oracle_mod):
    """test_solver_xpbd.py:149-225: friction reduces the tangential slip of one step."""

    def slip(mu):
        m = _two_particles((0.0, 0.0, 10.0), (0.0, 0.0, 0.0), mu)
        md = _model_dict(m)
        _, _, xo, _ = oracle_mod.xpbd_particle_step(md, m.particle_q.numpy(), m.particle_qd.numpy(),
                                                    np.zeros((2, 3), np.float32), 1.0 / 30.0, 30, 0.9)
        return float(abs(xo[0, 2] - xo[1, 2]))

    s0, s1 = slip(0.0), slip(1.0)
    assert s0 > 0.2
    assert s1 < 0.95 * s0


def test_reference_restitution_correct_particle(oracle_mod):
    """test_solver_xpbd.py:228-297: restitution goes to the contacting particle."""
    import newton_sph_dev_b200 as nsph

    b = nsph.ModelBuilder(up_axis="Y")
    b.add_particle(pos=(0.0, 10.0, 0.0), vel=(0.0, 0.0, 0.0), mass=1.0, radius=0.1)
    b.add_particle(pos=(0.0, 0.1, 0.0), vel=(0.0, -5.0, 0.0), mass=1.0, radius=0.1)
    b.add_ground_plane()
    m = b.finalize("cpu")
    m.set_gravity((0.0, 0.0, 0.0))
    m.soft_contact_restitution = 1.0
    md = _model_dict(m)
    x, v = m.particle_q.numpy(), m.particle_qd.numpy()
    c = oracle_mod.soft_contacts_create(md["shapes"], x, md["radius"], md["flags"], world=md["world"], margin=0.01)
    _, _, xo, vo = oracle_mod.xpbd_particle_step(md, x, v, np.zeros((2, 3), np.float32), 1.0 / 60.0, 10, 0.9,
                                                 contacts=c, enable_restitution=True)
    assert abs(vo[0, 1]) < 5e-3
    assert vo[1, 1] > 0.0
