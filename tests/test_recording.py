"""State dumps, trajectory recording and JSONL metrics, on the CPU."""

from __future__ import annotations

import numpy as np
import pytest
import torch


def _model():
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    b = nsph.ModelBuilder()
    SolverSPH.register_custom_attributes(b)
    b.add_particle_grid(pos=(0.005, 0.005, 0.005), rot=(0, 0, 0, 1), vel=(0.1, 0, 0), dim_x=6, dim_y=5, dim_z=4,
                        cell_x=0.01, cell_y=0.01, cell_z=0.01, mass=1e-3, jitter=0.002)
    return b.finalize("cpu")


def test_state_round_trip(tmp_path):
    from newton_sph_dev_b200 import recording

    m = _model()
    s = m.state()
    s.particle_f.normal_()
    s.sph.density.fill_(1003.5)
    p = recording.save_state(tmp_path / "state", s, step=17, sim_time=1.7e-3, scene="grid")
    assert p.name == "state.npz" and p.exists()
    s2 = m.state()
    info = recording.load_state(p, s2)
    assert info["step"] == 17 and info["scene"] == "grid" and abs(info["sim_time"] - 1.7e-3) < 1e-12
    for name in ("particle_q", "particle_qd", "particle_f"):
        assert torch.equal(getattr(s2, name), getattr(s, name)), name
    assert torch.equal(s2.sph.density, s.sph.density)
    arrays, _ = recording.read_state_file(p)
    assert "sph.density" in arrays


def test_state_load_refuses_other_shapes(tmp_path):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200 import recording

    m = _model()
    p = recording.save_state(tmp_path / "s.npz", m.state())
    b = nsph.ModelBuilder()
    b.add_particle((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 1.0)
    other = b.finalize("cpu").state()
    with pytest.raises(ValueError):
        recording.load_state(p, other)  # arrays differ (no sph namespace)
    with pytest.raises(ValueError):
        recording.load_state(p, other, strict=False)  # particle_q shape differs
    np.savez(tmp_path / "x.npz", __meta__=np.array('{"format": "something else"}'))
    with pytest.raises(ValueError):
        recording.read_state_file(tmp_path / "x.npz")


def test_trajectory_recorder(tmp_path):
    from newton_sph_dev_b200 import recording

    m = _model()
    s = m.state()
    rec = recording.TrajectoryRecorder(tmp_path / "traj.npz", every=3, arrays=("particle_q", "sph.density"),
                                       max_frames=4)
    kept = []
    for k in range(10):
        s.particle_q.add_(0.001)
        s.sph.density.fill_(float(k))
        if rec.record(s, step=100 + k):
            kept.append(k)
    assert kept == [0, 3, 6, 9] and len(rec) == 4
    with pytest.raises(RuntimeError):
        for _ in range(3):
            rec.record(s)
    path = rec.save(dt=1e-4)
    frames, steps, info = recording.TrajectoryRecorder.load(path)
    assert steps.tolist() == [100, 103, 106, 109] and info["every"] == 3 and info["dt"] == 1e-4
    assert frames["particle_q"].shape == (4, m.particle_count, 3)
    assert frames["sph.density"][:, 0].tolist() == [0.0, 3.0, 6.0, 9.0]
    np.testing.assert_allclose(frames["particle_q"][1] - frames["particle_q"][0], 0.003, atol=1e-6)
    with pytest.raises(KeyError):
        recording.TrajectoryRecorder(tmp_path / "t2", arrays=("nope",)).record(s)
    with pytest.raises(ValueError):
        recording.TrajectoryRecorder(tmp_path / "t3", every=0)


def test_metrics_log(tmp_path):
    from newton_sph_dev_b200 import recording

    path = tmp_path / "m.jsonl"
    with recording.MetricsLog(path) as log:
        log.log(step=1, rate=1.8e9, compression=torch.tensor(0.004), worst=np.float32(0.01))
        log.log(step=2, fallbacks=0, window=np.arange(3))
    with recording.MetricsLog(path) as log:  # appends
        log.log(step=3)
    recs = recording.MetricsLog.read(path)
    assert [r["step"] for r in recs] == [1, 2, 3]
    assert abs(recs[0]["compression"] - 0.004) < 1e-9 and recs[1]["window"] == [0, 1, 2]
    assert all("time" in r for r in recs)


def test_training_data_round_trip(tmp_path):
    from newton_sph_dev_b200.train_surrogate import load_training_data, save_training_data

    f = torch.randn(50, 16)
    t = torch.randn(50, 3)
    save_training_data(tmp_path / "d.npz", f, t, {"trajectories": 2, "dt": 1e-4})
    f2, t2, info = load_training_data(tmp_path / "d.npz", "cpu")
    assert torch.equal(f, f2) and torch.equal(t, t2) and info["trajectories"] == 2
    save_training_data(tmp_path / "bad.npz", f, t[:10], {})
    with pytest.raises(ValueError):
        load_training_data(tmp_path / "bad.npz", "cpu")


@pytest.mark.gpu
def test_resume_from_dump_is_bit_exact(tmp_path):
    """Ten SPH steps, a dump, ten more; a fresh solver and state loaded from
    the dump reach the same final state bit for bit."""
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200 import recording
    from newton_sph_dev_b200.solvers import SolverSPH

    b = nsph.ModelBuilder()
    SolverSPH.register_custom_attributes(b)
    b.add_particle_grid(pos=(0.005, 0.005, 0.005), rot=(0, 0, 0, 1), vel=(0.0, 0.0, 0.0), dim_x=24, dim_y=24,
                        dim_z=24, cell_x=0.01, cell_y=0.01, cell_z=0.01, mass=1e-3, jitter=0.002)
    m = b.finalize("cuda:0")
    cfg = SolverSPH.Config(smoothing_length=0.02, box_lo=(0.0, 0.0, 0.0), box_hi=(0.5, 0.5, 0.5))
    dt = 1e-4

    def run(solver, s0, s1, steps):
        for _ in range(steps):
            solver.step(s0, s1, None, None, dt)
            s0, s1 = s1, s0
        return s0, s1

    solver = SolverSPH(m, cfg)
    s0, s1 = run(solver, m.state(), m.state(), 10)
    path = recording.save_state(tmp_path / "mid", s0, step=10)
    a0, _ = run(solver, s0, s1, 10)
    r0 = m.state()
    recording.load_state(path, r0)
    b0, _ = run(SolverSPH(m, cfg), r0, m.state(), 10)
    torch.cuda.synchronize()
    assert torch.equal(a0.particle_q, b0.particle_q) and torch.equal(a0.particle_qd, b0.particle_qd)
    assert torch.equal(a0.sph.density, b0.sph.density)
