"""The fp32 restatement of the particle raycast depth camera
(oracle/raycast.c): the reference's own known answers for particles
(newton/tests/test_sensor_raycast.py:185-356), the C loop against a
pure-Python restatement of the same loop (grid aliasing, zero and negative
radii, hits and misses), an fp64 geometric pin of the depths, and the host
helpers of SensorRaycast (camera basis, march-step count). CPU only."""

from __future__ import annotations

import math

import numpy as np
import pytest

DIMS = (128, 128, 128)


def camera(oracle_mod, position, direction, up, fov, width, height, max_distance):
    from newton_sph_dev_b200.sensors import camera_basis

    d, u, r = camera_basis(direction, up)
    return oracle_mod.raycast_camera(position, d, u, r, math.tan(fov * 0.5), float(width) / float(height), width,
                                     height, max_distance)


def render(oracle_mod, x, radius, cam, step=None, dims=DIMS):
    from newton_sph_dev_b200.sensors import march_steps

    sr = float(np.max(radius)) + 1e-6
    step = 0.5 * sr if step is None else step
    max_steps = march_steps(cam.max_distance, step)[0]
    return oracle_mod.raycast_particles(x, radius, dims, cam, sr, step, max_steps)


def test_particle_hit_like_the_reference(oracle_mod):
    """test_sensor_raycast_particles_hit: a particle of radius 0.5 at
    (0, 0, 2) seen from the origin along +Z gives depth 1.5."""
    cam = camera(oracle_mod, (0, 0, 0), (0, 0, 1), (0, 1, 0), 0.1, 1, 1, 10.0)
    depth = render(oracle_mod, [[0.0, 0.0, 2.0]], [0.5], cam)
    assert depth.shape == (1, 1)
    assert depth[0, 0] > 0.0
    assert abs(float(depth[0, 0]) - 1.5) <= 1e-3


def test_no_particles_no_hit(oracle_mod):
    """test_sensor_raycast_include_particles_without_particles: -1."""
    cam = camera(oracle_mod, (0, 0, 0), (0, 0, 1), (0, 1, 0), 0.1, 1, 1, 5.0)
    depth = oracle_mod.raycast_particles(np.zeros((0, 3)), np.zeros(0), DIMS, cam, 0.1, 0.05, 100)
    assert depth[0, 0] == -1.0


def test_closest_particle_wins_and_max_distance(oracle_mod):
    cam = camera(oracle_mod, (0, 0, 0), (0, 0, 1), (0, 1, 0), 0.1, 1, 1, 10.0)
    depth = render(oracle_mod, [[0.0, 0.0, 6.0], [0.0, 0.0, 3.0]], [0.5, 0.5], cam)
    assert abs(float(depth[0, 0]) - 2.5) <= 1e-3
    # beyond max_distance: no hit
    cam = camera(oracle_mod, (0, 0, 0), (0, 0, 1), (0, 1, 0), 0.1, 1, 1, 2.0)
    depth = render(oracle_mod, [[0.0, 0.0, 6.0]], [0.5], cam)
    assert depth[0, 0] == -1.0


def _scene(seed, n, spread=0.4, center=(0.0, 0.0, 1.0)):
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-spread, spread, (n, 3)) + np.asarray(center)).astype(np.float32)
    r = rng.uniform(0.02, 0.08, n).astype(np.float32)
    r[::7] = 0.0  # skipped by the kernel
    r[3::11] = -0.05
    return x, r


@pytest.mark.parametrize("dims", [(128, 128, 128), (5, 4, 3)])
def test_c_loop_equals_python_loop(oracle_mod, dims):
    """raycast.c and the pure-Python loop agree bit for bit, with a grid that
    aliases far cells onto the same physical cells (dims 5 x 4 x 3) and one
    that does not."""
    x, r = _scene(3, 150, spread=0.3)
    cam = camera(oracle_mod, (0.05, -0.1, -1.0), (0.0, 0.05, 1.0), (0, 1, 0), 0.45, 7, 5, 4.0)
    sr = float(np.max(r)) + 1e-6
    step = 0.5 * sr
    from newton_sph_dev_b200.sensors import march_steps

    steps = march_steps(cam.max_distance, step)[0]
    got = oracle_mod.raycast_particles(x, r, dims, cam, sr, step, steps)
    ref = oracle_mod.raycast_particles_py(x, r, dims, cam, sr, step, steps)
    np.testing.assert_array_equal(got, ref)
    assert (got > 0).sum() >= 5 and (got < 0).sum() >= 1  # hits and misses both occur


def test_depths_match_fp64_geometry(oracle_mod):
    """Where the ray passes well inside a sphere (not grazing it, where the
    march can step past), the depth is the fp64 distance to the nearest
    sphere surface along the ray."""
    x, r = _scene(5, 200)
    r = np.abs(r)
    r[r == 0] = 0.03
    cam = camera(oracle_mod, (0.0, 0.0, -1.0), (0.0, 0.0, 1.0), (0, 1, 0), 1.0, 40, 30, 4.0)
    depth = render(oracle_mod, x, r, cam)
    from newton_sph_dev_b200.sensors import camera_basis

    d, u, rt = camera_basis((0.0, 0.0, 1.0), (0, 1, 0))
    checked = 0
    for py in range(cam.height):
        for px in range(cam.width):
            ndc_x = (2.0 * px + 1.0) / cam.width - 1.0
            ndc_y = 1.0 - (2.0 * py + 1.0) / cam.height
            dirv = rt.astype(np.float64) * ndc_x * cam.fov_scale * cam.aspect_ratio + \
                u.astype(np.float64) * ndc_y * cam.fov_scale + d.astype(np.float64)
            dirv /= np.linalg.norm(dirv)
            o = np.array(cam.position[:], np.float64)
            oc = o - x.astype(np.float64)
            proj = oc @ dirv
            disc = proj * proj - (np.sum(oc * oc, axis=1) - r.astype(np.float64) ** 2)
            ok = disc > 0
            t = np.where(ok, -proj - np.sqrt(np.where(ok, disc, 0.0)), np.inf)
            t[t < 0] = np.inf
            k = int(np.argmin(t))
            if not np.isfinite(t[k]):
                continue
            miss = np.sqrt(max(0.0, float(np.sum(oc[k] * oc[k]) - proj[k] ** 2)))  # ray-centre distance
            if miss > 0.5 * r[k]:
                continue  # grazing: the march may legitimately step past
            assert abs(float(depth[py, px]) - t[k]) <= 1e-5 * max(1.0, t[k]), (py, px)
            checked += 1
    assert checked >= 20


def test_march_steps_like_the_reference():
    from newton_sph_dev_b200.sensors import MAX_PARTICLE_RAY_MARCH_STEPS, march_steps

    assert march_steps(10.0, 0.25) == (41, False, 41)
    steps, truncated, requested = march_steps(1.0e12, 1.0e-9)
    assert truncated and steps == MAX_PARTICLE_RAY_MARCH_STEPS and requested > steps
    assert march_steps(float("inf"), 1.0)[1]
    with pytest.raises(ValueError):
        march_steps(10.0, 0.0)


def test_camera_basis_is_orthonormal_and_handles_parallel_up():
    from newton_sph_dev_b200.sensors import camera_basis

    for direction, up in (((1, 0, 0), (0, 0, 1)), ((0.3, -2.0, 0.5), (0, 0, 5)), ((0, 0, 1), (0, 0, 1))):
        d, u, r = camera_basis(direction, up)
        m = np.stack([d, u, r]).astype(np.float64)
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-6)
        np.testing.assert_allclose(np.cross(d, u), r, atol=1e-6)
