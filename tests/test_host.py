"""Host-side logic of the Newton-compatible API (CPU only): builder ordering
and finalize (newton/_src/sim/builder.py:7186-7275, 8037-8130, 9815-9855),
worlds and gravity (:2815-2909, :10655-10668), State.assign / clear_forces
(newton/_src/sim/state.py:156-229), Model.set_gravity (model.py:923-956) and
the solver configuration (grid sizing, fp32 constants)."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import newton_sph_dev_b200 as nsph
from newton_sph_dev_b200 import ParticleFlags
from newton_sph_dev_b200.sim.builder import quat_to_matrix
from newton_sph_dev_b200.solvers import SolverNotifyFlags, SolverSPH


def test_add_particle_and_finalize_fields():
    b = nsph.ModelBuilder()
    i0 = b.add_particle((1, 2, 3), (0, 0, -1), mass=2.0)
    i1 = b.add_particle((4, 5, 6), (0, 0, 0), mass=0.0, radius=0.3, flags=0)
    assert (i0, i1) == (0, 1)
    m = b.finalize("cpu")
    assert m.particle_count == 2
    assert m.particle_q.dtype == torch.float32 and tuple(m.particle_q.shape) == (2, 3)
    assert m.particle_inv_mass.tolist() == [0.5, 0.0]
    assert m.particle_radius.tolist() == pytest.approx([0.1, 0.3])
    assert m.particle_flags.tolist() == [int(ParticleFlags.ACTIVE), 0]
    assert m.particle_world.tolist() == [-1, -1]
    assert m.particle_max_radius == pytest.approx(0.3)
    assert m.particle_max_velocity == 1e5
    assert m.world_count == 1
    assert m.gravity.tolist() == [[0.0, 0.0, pytest.approx(-9.81)]]
    assert m.particle_grid is None  # CPU model: no device grid


def test_up_axis_and_world_gravity():
    b = nsph.ModelBuilder(up_axis=1, gravity=-3.0)
    b.begin_world()
    b.add_particle((0, 0, 0), (0, 0, 0), 1.0)
    b.end_world()
    b.begin_world(gravity=(1.0, 2.0, 3.0))
    b.add_particle((0, 0, 0), (0, 0, 0), 1.0)
    b.add_particle((0, 0, 0), (0, 0, 0), 1.0)
    b.end_world()
    b.add_particle((0, 0, 0), (0, 0, 0), 1.0)
    with pytest.raises(RuntimeError):
        b.end_world()
    m = b.finalize("cpu")
    assert m.world_count == 2
    assert m.gravity.tolist() == [[0.0, -3.0, 0.0], [1.0, 2.0, 3.0]]
    assert m.particle_world.tolist() == [0, 1, 1, -1]
    assert m.particle_world_start.tolist() == [0, 1, 3, 4]


def test_particle_grid_order_and_seed():
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(0, 0, 0), rot=(0, 0, 0, 1), vel=(1, 2, 3), dim_x=3, dim_y=2, dim_z=4, cell_x=1.0,
                        cell_y=10.0, cell_z=100.0, mass=0.5, jitter=0.0)
    q = b.particle_q
    # index = iy*(dim_x*dim_z) + ix*dim_z + iz
    for iy in range(2):
        for ix in range(3):
            for iz in range(4):
                assert q[iy * 12 + ix * 4 + iz].tolist() == [ix * 1.0, iy * 10.0, iz * 100.0]
    assert np.all(b.particle_qd == [1, 2, 3])
    m = b.finalize("cpu")
    assert m.particle_q.is_contiguous() and m.particle_qd.is_contiguous()
    # jitter stream: default_rng(42 + particle_count) over the (N, 3) array
    b2 = nsph.ModelBuilder()
    b2.add_particle_grid(pos=(0, 0, 0), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=3, dim_y=2, dim_z=4, cell_x=1.0,
                         cell_y=10.0, cell_z=100.0, mass=0.5, jitter=0.2)
    rng = np.random.default_rng(42)
    assert np.array_equal(b2.particle_q, q + (rng.random((24, 3)) - 0.5) * 0.2)


def test_particle_grid_rotation():
    r = quat_to_matrix((0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4)))  # 90 deg about z
    assert np.allclose(r @ np.array([1.0, 0.0, 0.0]), [0.0, 1.0, 0.0], atol=1e-6)
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(10, 0, 0), rot=(0.0, 0.0, math.sin(math.pi / 4), math.cos(math.pi / 4)),
                        vel=(0, 0, 0), dim_x=2, dim_y=1, dim_z=1, cell_x=1.0, cell_y=1.0, cell_z=1.0, mass=1.0,
                        jitter=0.0)
    assert np.allclose(b.particle_q, [[10, 0, 0], [10, 1, 0]], atol=1e-6)


def test_radius_std_and_flags():
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(0, 0, 0), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=4, dim_y=4, dim_z=4, cell_x=1, cell_y=1,
                        cell_z=1, mass=1.0, jitter=0.1, radius_mean=0.5, radius_std=0.01, flags=0)
    assert np.all(b.particle_flags == 0)
    rng = np.random.default_rng(42)
    rng.random((64, 3))
    assert np.array_equal(b.particle_radius, 0.5 + rng.standard_normal(64) * 0.01)
    with pytest.raises(ValueError):
        b.add_particle_grid(pos=(0, 0, 0), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=2, dim_y=1, dim_z=1, cell_x=1,
                            cell_y=1, cell_z=1, mass=1.0, jitter=0.0, flags=[1, 1, 1])


def test_state_assign_and_clear_forces():
    b = nsph.ModelBuilder()
    SolverSPH.register_custom_attributes(b)
    b.add_particle((0, 0, 0), (1, 1, 1), 1.0)
    m = b.finalize("cpu")
    s0, s1 = m.state(), m.state()
    assert s0.sph.density.shape == (1,)
    s1.particle_q.fill_(5.0)
    s1.sph.density.fill_(7.0)
    s0.assign(s1)
    assert s0.particle_q.tolist() == [[5.0, 5.0, 5.0]] and s0.sph.density.tolist() == [7.0]
    s0.particle_f.fill_(3.0)
    s0.clear_forces()
    assert s0.particle_f.abs().sum() == 0
    s2 = nsph.State()
    s2.particle_q = torch.zeros(1, 3)
    with pytest.raises(ValueError):
        s0.assign(s2)
    s3 = m.state()
    del s3.sph
    with pytest.raises(ValueError):
        s0.assign(s3)


def test_set_gravity_variants():
    b = nsph.ModelBuilder()
    b.begin_world()
    b.end_world()
    b.begin_world()
    b.end_world()
    m = b.finalize("cpu")
    m.set_gravity((0.0, 1.0, 0.0))
    assert m.gravity.tolist() == [[0, 1, 0], [0, 1, 0]]
    m.set_gravity((0.0, 0.0, 2.0), world=1)
    assert m.gravity.tolist() == [[0, 1, 0], [0, 0, 2]]
    m.set_gravity([[1, 1, 1], [2, 2, 2]])
    assert m.gravity.tolist() == [[1, 1, 1], [2, 2, 2]]
    with pytest.raises(IndexError):
        m.set_gravity((0, 0, 0), world=2)
    with pytest.raises(ValueError):
        m.set_gravity([[1, 1, 1]] * 3)
    assert SolverNotifyFlags.MODEL_PROPERTIES == 1 << 5


def test_config_constants_are_fp32_exact():
    cfg = SolverSPH.Config(smoothing_length=0.01)
    c = cfg.constants(5e-5, 1e5)["f32"]
    assert c["h2"] == np.float32(np.float32(0.01) * np.float32(0.01))
    assert c["cell_inv"] == np.float32(1.0) / np.float32(0.01)
    assert c["eos_b"] == np.float32(1000 * 400 / 7)
    h = float(np.float32(0.01))
    assert c["sigma"] == np.float32(8 / (math.pi * h**3))
    p = cfg.params(5e-5, 1e5)
    assert p.h == pytest.approx(0.01) and p.eos_gamma == 7 and p.dt == pytest.approx(5e-5)


@pytest.mark.parametrize("box,h,expect", [((1, 1, 1), 0.02, (64, 64, 64)), ((2, 1, 1), 0.01, (256, 128, 128)),
                                          ((0.5, 0.5, 0.5), 0.008, (128, 128, 128))])
def test_grid_dims_cover_the_box(box, h, expect):
    cfg = SolverSPH.Config(smoothing_length=h, box_lo=(0, 0, 0), box_hi=box)
    dims = cfg.resolved_grid_dims()
    assert dims == expect
    inv = np.float32(1.0) / np.float32(h)
    for a in range(3):
        # cells -1 .. int(hi*inv)+1 map to distinct physical cells
        span = int(np.float32(np.float32(box[a]) * inv)) + 3
        assert dims[a] >= span and dims[a] & (dims[a] - 1) == 0


def test_default_grid_without_box_is_128_cubed():
    assert SolverSPH.Config(smoothing_length=0.1).resolved_grid_dims() == (128, 128, 128)
