"""The particle raycast depth camera on the GPU (nsph_raycast_particles,
SensorRaycast): bit-exact against the oracle's restatement of the
reference's loop (oracle/raycast.c, which queries every cell at every march
sample, so it also checks that the device's once-per-cell visiting is
exact), with a grid that aliases and one that does not and with depths
already present (shape hits); and the reference's known answers for
particles (newton/tests/test_sensor_raycast.py:185-356)."""

from __future__ import annotations

import ctypes
import math
import warnings

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _camera(oracle_mod, position, direction, up, fov, width, height, max_distance):
    from newton_sph_dev_b200 import _lib
    from newton_sph_dev_b200.sensors import camera_basis

    d, u, r = camera_basis(direction, up)
    args = (position, d, u, r, math.tan(fov * 0.5), float(width) / float(height), width, height, max_distance)
    c = _lib.NsphRaycastCamera()
    c.position[:], c.direction[:], c.up[:], c.right[:] = [[float(np.float32(v)) for v in a] for a in args[:4]]
    c.fov_scale, c.aspect_ratio = float(np.float32(args[4])), float(np.float32(args[5]))
    c.width, c.height, c.max_distance = width, height, float(np.float32(max_distance))
    return c, oracle_mod.raycast_camera(*args)


def _device_depth(x, r, dims, cam, sr, step, steps, depth_init):
    from newton_sph_dev_b200 import HashGrid, _lib

    xt = torch.from_numpy(x).to(DEV)
    rt = torch.from_numpy(r).to(DEV)
    grid = HashGrid(*dims, device=DEV)
    grid.reserve(len(x))
    grid.build(xt, sr)
    depth = torch.from_numpy(depth_init.copy()).to(DEV)
    L = _lib.load()
    st = L.nsph_raycast_particles(grid.id, xt.data_ptr(), rt.data_ptr(), len(x), ctypes.byref(cam), float(sr),
                                  float(step), int(steps), depth.data_ptr(), _lib.stream_handle(torch.device(DEV)))
    _lib.check(st, "raycast")
    raw = depth.cpu().numpy()
    _lib.check(L.nsph_raycast_clamp_no_hits(depth.data_ptr(), depth.numel(), float(cam.max_distance),
                                            _lib.stream_handle(torch.device(DEV))), "clamp")
    return raw, depth.cpu().numpy()


@pytest.mark.parametrize("dims", [(128, 128, 128), (7, 5, 6)])
def test_device_equals_oracle(oracle_mod, dims):
    from newton_sph_dev_b200.sensors import march_steps

    rng = np.random.default_rng(11)
    n = 3000
    x = (rng.uniform(-0.5, 0.5, (n, 3)) + [0.0, 0.0, 1.5]).astype(np.float32)
    r = rng.uniform(0.005, 0.03, n).astype(np.float32)
    r[::13] = 0.0
    r[5::17] = -0.01
    cam, ocam = _camera(oracle_mod, (0.1, 0.05, -0.8), (0.0, -0.02, 1.0), (0, 1, 0), 0.9, 64, 48, 4.0)
    sr = float(r.max()) + 1e-6
    step = 0.5 * sr
    steps = march_steps(4.0, step)[0]
    init = np.full((48, 64), np.float32(4.0), np.float32)
    init[::5, ::3] = rng.uniform(0.5, 4.5, init[::5, ::3].shape).astype(np.float32)  # shape hits present
    init[1::7, 2::9] = -1.0
    raw, clamped = _device_depth(x, r, dims, cam, sr, step, steps, init)
    ref_raw = oracle_mod.raycast_particles(x, r, dims, ocam, sr, step, steps, depth_init=init, clamp=False)
    np.testing.assert_array_equal(raw, ref_raw)
    ref = ref_raw.copy()
    oracle_mod.lib().oracle_raycast_clamp_no_hits(ref.ctypes.data, ref.size, ocam.max_distance)
    np.testing.assert_array_equal(clamped, ref)
    hits = (clamped > 0) & (init >= 4.0)
    assert hits.sum() > 200 and (clamped < 0).sum() > 10


def test_lattice_block_equals_oracle(oracle_mod):
    """A 100k-particle lattice block (spheres touching) seen at an angle,
    through SensorRaycast, against the oracle."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.sensors import SensorRaycast, march_steps

    g = np.stack(np.meshgrid(*[np.arange(k) for k in (50, 50, 40)], indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(2)
    x = ((g + 0.5) * 0.01 + rng.uniform(-0.001, 0.001, g.shape)).astype(np.float32)
    r = np.full(len(x), 0.005, np.float32)
    b = nsph.ModelBuilder()
    b.add_particles(pos=x.tolist(), vel=np.zeros_like(x).tolist(), mass=[1.0] * len(x), radius=r.tolist())
    model = b.finalize(DEV)
    state = model.state()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", DeprecationWarning)
        sensor = SensorRaycast(model, (1.2, -0.6, 0.9), (-0.8, 0.8, -0.4), (0, 0, 1), 0.8, 96, 72, max_distance=3.0)
    sensor.update(state, include_particles=True)
    got = sensor.get_depth_image_numpy()
    ocam = oracle_mod.raycast_camera(sensor.camera_position, sensor.camera_direction, sensor.camera_up,
                                     sensor.camera_right, sensor.fov_scale, sensor.aspect_ratio, 96, 72, 3.0)
    sr = 0.005 + 1e-6
    ref = oracle_mod.raycast_particles(x, r, (128, 128, 128), ocam, sr, 0.5 * sr, march_steps(3.0, 0.5 * sr)[0])
    np.testing.assert_array_equal(got, ref)
    assert (got > 0).sum() > 1000 and (got < 0).sum() > 100


def _one_particle_sensor(radius=0.5, max_distance=10.0, with_particle=True):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.sensors import SensorRaycast

    b = nsph.ModelBuilder()
    if with_particle:
        b.add_particle(pos=(0.0, 0.0, 2.0), vel=(0.0, 0.0, 0.0), mass=0.0, radius=radius)
    model = b.finalize(DEV)
    state = model.state()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", DeprecationWarning)
        sensor = SensorRaycast(model, (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 0.1, 1, 1,
                               max_distance=max_distance)
    return sensor, state


def test_reference_known_answers():
    # test_sensor_raycast_particles_hit
    sensor, state = _one_particle_sensor()
    sensor.update(state, include_particles=True)
    depth = sensor.get_depth_image_numpy()
    assert depth.shape == (1, 1) and depth[0, 0] > 0.0 and abs(float(depth[0, 0]) - 1.5) <= 1e-3
    # particles are off by default: no hit
    sensor.update(state)
    assert sensor.get_depth_image_numpy()[0, 0] == -1.0
    # test_sensor_raycast_particles_requires_positive_step
    with pytest.raises(ValueError):
        sensor.update(state, include_particles=True, particle_march_step=0.0)
    # test_sensor_raycast_include_particles_without_particles
    sensor, state = _one_particle_sensor(max_distance=5.0, with_particle=False)
    sensor.update(state, include_particles=True)
    assert sensor.get_depth_image_numpy()[0, 0] == -1.0
    # test_sensor_raycast_particle_step_truncation_warns
    sensor, state = _one_particle_sensor(radius=0.1, max_distance=1.0e12)
    with pytest.warns(RuntimeWarning):
        sensor.update(state, include_particles=True, particle_march_step=1.0e-9)


def test_deprecation_and_camera_setters():
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.sensors import SensorRaycast

    b = nsph.ModelBuilder()
    b.add_particle(pos=(5.0, 1.0, 0.5), vel=(0.0, 0.0, 0.0), mass=1.0, radius=0.2)
    model = b.finalize(DEV)
    with pytest.warns(DeprecationWarning):
        sensor = SensorRaycast(model, (0, 0, 0), (1, 0, 0), (0, 0, 1), 1.6, 3, 3, max_distance=20.0)
    # like test_sensor_raycast_single_pixel_hit, with a particle for the sphere
    sensor.point_camera_at(target=(5.0, 1.0, 0.5), position=(0, 0, 0), up=(0, 0, 1))
    sensor.update(model.state(), include_particles=True)
    depth = sensor.get_depth_image_numpy()
    hits = np.argwhere(depth > 0.0)
    assert hits.shape[0] == 1 and tuple(hits[0]) == (1, 1)
    assert abs(float(depth[1, 1]) - (np.linalg.norm([5.0, 1.0, 0.5]) - 0.2)) <= 1e-3
    sensor.update_camera_parameters(width=8, height=4, max_distance=30.0)
    assert sensor.get_depth_image().shape == (4, 8) and sensor.aspect_ratio == 2.0
    sensor.update(model.state(), include_particles=True)
    assert sensor.get_depth_image_numpy().shape == (4, 8)
