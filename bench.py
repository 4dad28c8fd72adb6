#!/usr/bin/env python
"""Throughput of the plain WCSPH step: particle-steps/s at 1M particles.

Workload (default ``tank_1m``): 1,048,576 fp32 particles as a 128x128x64
jittered lattice block (spacing 0.005 m, jitter +-0.1 spacing, seed rule of
ModelBuilder.add_particle_grid) in the corner of a 2x1x1 m tank, initial
velocities N(0, 0.01 m/s) per component (numpy default_rng(2)), h = 2 x
spacing, rho0 = 1000, Tait gamma = 7, c0 = 20 m/s, XSPH 0.01, gravity -9.81,
dt = 5e-5 s. Synthetic data, generated on the host like the reference's
builder.

One step = one SolverSPH.step (grid build, density/EOS pass,
force/XSPH/integrate pass), replayed from a CUDA graph captured per step.
Between timed steps L2 is flushed by writing a 256 MiB buffer (outside the
timed intervals); each step is timed on the device with CUDA events recorded
inside the graph, which also split it into build / density / force phases.

Multi-GPU: the step does not shard (a single scene); ``--gpus N`` runs N
independent replicas, one per rank, timed as the max over ranks.

``--impl reference`` times the CPU restatement of the path (the oracle,
OpenMP on all host cores) on the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

METRIC = "particle-steps/s"
B_ALG_STEP = 64  # algorithmic HBM bytes per particle-step (read x,v 24 + write x,v 24 + density 8 + cell key 8)
# algorithmic bytes per particle of each single-kernel pass (unique data it must move)
B_ALG_DENSITY = 12 + 8  # read x; write (m/rho, p/rho^2)
B_ALG_FORCE = 24 + 8 + 24  # read x, v; read density scratch; write x, v

WORKLOADS = {
    "tank_1m": dict(shape=(128, 128, 64), spacing=0.005, box=(2.0, 1.0, 1.0), dt=5e-5, vel_std=0.01,
                    desc="1,048,576 particles, 128x128x64 block at 0.005 m in a 2x1x1 m tank"),
    "tank_2m": dict(shape=(128, 128, 128), spacing=0.005, box=(2.0, 1.0, 1.0), dt=5e-5, vel_std=0.01,
                    desc="2,097,152 particles, 128^3 block at 0.005 m in a 2x1x1 m tank"),
    "dam_break_32k": dict(shape=(32, 32, 32), spacing=0.01, box=(1.0, 1.0, 1.0), dt=1e-4, vel_std=0.0,
                          desc="32,768 particles, 32^3 block at 0.01 m in a 1 m box"),
    "rollout_grad_64k": dict(shape=(64, 64, 16), spacing=0.01, box=(1.0, 1.0, 1.0), dt=1e-4, vel_std=0.1, vel_seed=4,
                             grad=dict(steps=50, checkpoint=10, target_seed=5),
                             desc="differentiable rollout: 65,536 particles (64x64x16 block at 0.01 m in a 1 m box), "
                                  "v0 ~ N(0, 0.1 m/s), 50 steps at dt = 1e-4 s, loss = mean |x_T - y|^2 against a "
                                  "seeded target cloud, gradients w.r.t. x0, v0 and the EOS stiffness B, checkpoint "
                                  "every 10 steps"),
    "tank_1m_surrogate": dict(shape=(128, 128, 64), spacing=0.005, box=(2.0, 1.0, 1.0), dt=5e-5, vel_std=0.01,
                              surrogate=dict(substeps=4, threshold=0.01, window=10),
                              metric="effective particle-steps/s",
                              desc="learned surrogate on the 1,048,576-particle tank: one step of 4 x 5e-5 s with "
                                   "the MLP acceleration correction (tcgen05) per call; a window of 10 calls whose "
                                   "compression error exceeds 1% is replaced by plain steps from its start, and the "
                                   "next window(s) run plain steps"),
    "tank_1m_surrogate_8x": dict(shape=(128, 128, 64), spacing=0.005, box=(2.0, 1.0, 1.0), dt=5e-5, vel_std=0.01,
                                 surrogate=dict(substeps=8, threshold=0.01, window=10,
                                                weights="surrogate_weights_8x.npz"),
                                 metric="effective particle-steps/s",
                                 desc="learned surrogate on the 1,048,576-particle tank at dt = 4e-4 s: one step of "
                                      "8 x 5e-5 s (dt c0 / h = 0.8) with the MLP correction per call; a window of 10 "
                                      "calls whose compression error exceeds 1% is replaced by plain steps from its "
                                      "start, and the next window(s) run plain steps (longer after failures in a row)"),
    "contact_1m": dict(shape=(128, 128, 64), spacing=0.0095, radius=0.005, vel_std=0.1, contact=True,
                       metric="particle-steps/s",
                       desc="particle-particle contact (eval_particle_contact): 1,048,576 spheres of radius 0.005 m "
                            "on a jittered 0.0095 m lattice (touching neighbours), v ~ N(0, 0.1 m/s); one step = "
                            "HashGrid build at 2 r_max + cohesion + contact forces"),
    "xpbd_1m": dict(shape=(128, 128, 64), spacing=0.0095, radius=0.005, vel_std=0.1, xpbd=dict(iterations=4, dt=1e-3),
                    metric="particle-steps/s",
                    desc="XPBD particle step (SolverXPBD): 1,048,576 spheres of radius 0.005 m on a jittered 0.0095 m "
                         "lattice resting on a ground plane, v ~ N(0, 0.1 m/s), gravity; one step = Model.collide "
                         "(soft contacts with the plane) + integrate + HashGrid build at 2 r_max + 4 iterations of "
                         "shape and particle corrections and apply_particle_deltas, dt = 1e-3 s"),
    "raycast_1m": dict(shape=(128, 128, 64), spacing=0.0095, radius=0.005, vel_std=0.0,
                       raycast=dict(width=640, height=480, fov=1.0, position=(2.2, -1.0, 1.6), target=(0.6, 0.6, 0.3),
                                    max_distance=4.0),
                       metric="rays/s",
                       desc="SensorRaycast particle depth image: 640x480 rays against 1,048,576 spheres of radius "
                            "0.005 m on a jittered 0.0095 m lattice (a 1.22 x 1.22 x 0.61 m block) seen from 2.6 m; "
                            "one step = HashGrid(128,128,128) build at r_max + 1e-6, the march (step half of that, "
                            "max distance 4 m) and the no-hit clamp"),
    "worlds_4096": dict(worlds=4096, n_range=(256, 16384), s_range=(0.004, 0.01), box=(0.5, 0.5, 0.5), dt=1e-4,
                        vel_std=0.0, seed=3,
                        desc="4,096 independent scenes: particles log-uniform in [256, 16384], spacing uniform in "
                             "[0.004, 0.01] m, h = 2 spacing, one jittered lattice block each in a 0.5 m cube"),
}


def worlds_layout(w):
    """Per-world (lattice dims, spacing) of the batched-worlds workload (seeded)."""
    rng = np.random.default_rng(w["seed"])
    lo, hi = w["n_range"]
    counts = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), w["worlds"]))).astype(int)
    spacing = rng.uniform(w["s_range"][0], w["s_range"][1], w["worlds"])
    out = []
    for nk, s in zip(counts, spacing):
        a = max(2, int(np.floor(nk ** (1.0 / 3.0))))
        c = max(1, int(round(nk / (a * a))))
        out.append(((a, a, c), float(s)))
    return out


def partition_worlds(sizes, parts: int) -> list[list[int]]:
    """Split worlds over `parts` ranks by particle count: largest first, each
    to the least-loaded rank (ties to the lowest rank); each rank keeps its
    worlds in their original order. Deterministic, so every rank computes the
    same split without communication."""
    loads = [0] * parts
    out = [[] for _ in range(parts)]
    for k in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(parts), key=lambda j: (loads[j], j))
        out[r].append(k)
        loads[r] += int(sizes[k])
    return [sorted(o) for o in out]


def world_sizes(layout) -> list[int]:
    return [a * b * c for (a, b, c), _ in layout]


def make_worlds_scene(name: str, device: str, max_worlds: int | None = None, subset: list[int] | None = None):
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    w = WORKLOADS[name]
    layout = worlds_layout(w)
    if max_worlds is not None:
        layout = layout[:max_worlds]
    if subset is not None:  # this rank's share of the worlds
        layout = [layout[k] for k in subset]
    b = nsph.ModelBuilder()
    cfgs = []
    for shape, s in layout:
        b.begin_world()
        b.add_particle_grid(pos=(s / 2, s / 2, s / 2), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=shape[0],
                            dim_y=shape[1], dim_z=shape[2], cell_x=s, cell_y=s, cell_z=s, mass=1000.0 * s**3,
                            jitter=0.2 * s)
        b.end_world()
        cfgs.append(SolverSPH.Config(smoothing_length=2 * s, rest_density=1000.0, sound_speed=20.0, eos_gamma=7,
                                     xsph=0.01, box_lo=(0.0, 0.0, 0.0), box_hi=w["box"]))
    model = b.finalize(device)
    return model, cfgs, w


def make_scene(name: str, device: str, rank: int = 0, world: int = 1):
    """The workload's scene; batched worlds are split over the ranks (each
    rank builds its share, see partition_worlds), other workloads are
    replicated."""
    import torch

    if "worlds" in WORKLOADS[name]:
        subset = None
        if world > 1:
            subset = partition_worlds(world_sizes(worlds_layout(WORKLOADS[name])), world)[rank]
        return make_worlds_scene(name, device, subset=subset)
    import newton_sph_dev_b200 as nsph
    from newton_sph_dev_b200.solvers import SolverSPH

    w = WORKLOADS[name]
    s = w["spacing"]
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(s / 2, s / 2, s / 2), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=w["shape"][0],
                        dim_y=w["shape"][1], dim_z=w["shape"][2], cell_x=s, cell_y=s, cell_z=s,
                        mass=1000.0 * s**3, jitter=0.2 * s)
    model = b.finalize(device)
    if w["vel_std"] > 0:
        rng = np.random.default_rng(seed=w.get("vel_seed", 2))
        v = rng.normal(0.0, w["vel_std"], (model.particle_count, 3)).astype(np.float32)
        model.particle_qd.copy_(torch.from_numpy(v))
    cfg = SolverSPH.Config(smoothing_length=2 * s, rest_density=1000.0, sound_speed=20.0, eos_gamma=7, xsph=0.01,
                           box_lo=(0.0, 0.0, 0.0), box_hi=w["box"])
    return model, cfg, w


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and clock-event reasons sampled during a timed region.

    NVML (pynvml) is polled from a thread every 2 ms, with one sample taken
    on entry and one on exit, so even a timed region of a few milliseconds
    carries a record. Without NVML, nvidia-smi's 20 ms loop is used."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu_index: int, period_s: float = 0.002):
        self.gpu_index = gpu_index
        self.period_s = period_s
        self.proc = None
        self.samples = []  # (sm_mhz, max_mhz, reason bits)
        self.lines = []
        self._nvml = None
        self._thread = None
        self._stop = None

    def _nvml_handle(self):
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.gpu_index).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            return None

    def _sample(self):
        nv, hdl = self._nvml
        try:
            sm = nv.nvmlDeviceGetClockInfo(hdl, nv.NVML_CLOCK_SM)
            mx = nv.nvmlDeviceGetMaxClockInfo(hdl, nv.NVML_CLOCK_SM)
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(hdl)
            self.samples.append((float(sm), float(mx), int(reasons)))
        except Exception:
            pass

    def __enter__(self):
        import threading

        self._nvml = self._nvml_handle()
        if self._nvml is not None:
            self._sample()
            self._stop = threading.Event()

            def loop():
                while not self._stop.wait(self.period_s):
                    self._sample()

            self._thread = threading.Thread(target=loop, daemon=True)
            self._thread.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join()
            self._sample()
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        for s, m, bits in self.samples:
            sm.append(s)
            mx = m
            for nm, bit in self.REASONS:
                if bits & bit:
                    reasons.add(nm)
        names = [nm for nm, _ in self.REASONS]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        src = "nvml" if self.samples else "nvidia-smi"
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0, "source": src}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": src}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas; timing = max over ranks)
# ---------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        if device is not None and device.type == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline (oracle restatement, all host threads)
# ---------------------------------------------------------------------------
def cpu_oracle_rate(model_cpu, cfg, w, budget_s: float, max_steps: int, sample_shape=None):
    """particle-steps/s of the oracle's fp32 step on the host cores."""
    from oracle import oracle as O

    O.build()
    if isinstance(cfg, list):  # batched worlds: one oracle step per world, on the first worlds
        x = model_cpu.particle_q.numpy()
        v = model_cpu.particle_qd.numpy()
        world = model_cpu.particle_world.numpy()
        m, inv = model_cpu.particle_mass.numpy(), model_cpu.particle_inv_mass.numpy()
        fl, g = model_cpu.particle_flags.numpy(), model_cpu.gravity.numpy()
        done = 0
        t0 = time.perf_counter()
        nw = 0
        for k, c in enumerate(cfg):
            sel = np.nonzero(world == k)[0]
            O.sph_step(c.constants(w["dt"], model_cpu.particle_max_velocity), c.resolved_grid_dims(tight=True),
                       x[sel], v[sel], m[sel], inv[sel], fl[sel], np.zeros(len(sel), np.int32), g[k:k + 1],
                       f_ext=np.zeros((len(sel), 3), np.float32), v_out_init=v[sel], precision="f32")
            done += len(sel)
            nw += 1
            if time.perf_counter() - t0 >= budget_s or nw >= max_steps:
                break
        el = time.perf_counter() - t0
        return done / el, nw, el, O.get_threads()
    x = model_cpu.particle_q.numpy()
    v = model_cpu.particle_qd.numpy()
    args = dict(mass=model_cpu.particle_mass.numpy(), inv_mass=model_cpu.particle_inv_mass.numpy(),
                flags=model_cpu.particle_flags.numpy(), world=model_cpu.particle_world.numpy(),
                gravity=model_cpu.gravity.numpy())
    consts = cfg.constants(w["dt"], model_cpu.particle_max_velocity)
    dims = cfg.resolved_grid_dims()
    f = np.zeros_like(x)
    steps = 0
    t0 = time.perf_counter()
    while True:
        r = O.sph_step(consts, dims, x, v, args["mass"], args["inv_mass"], args["flags"], args["world"],
                       args["gravity"], f_ext=f, v_out_init=v, precision="f32")
        x, v = r["x"], r["v"]
        steps += 1
        el = time.perf_counter() - t0
        if steps >= max_steps or el >= budget_s:
            break
    return x.shape[0] * steps / el, steps, el, O.get_threads()


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import torch  # noqa: F401

    name = args.workload
    model, cfg, w = make_scene(name, "cpu")
    n = model.particle_count
    from oracle import oracle as O

    O.build()
    # one untimed probe step sizes the sample so the whole run stays within a few minutes
    rate_probe, _, el, threads = cpu_oracle_rate(model, cfg, w, budget_s=0.0, max_steps=1)
    per_step = n / rate_probe
    total_steps = args.steps + args.warmup
    budget = 150.0
    sample_n = n
    sub = None
    if per_step * total_steps > budget:
        frac = budget / (per_step * total_steps)
        # cubic sub-block of the lattice with the same spacing
        k = max(8, int(round(min(w["shape"]) * frac ** (1 / 3))))
        sub = (min(k, w["shape"][0]), min(k, w["shape"][1]), min(k, w["shape"][2]))
        wsub = dict(w, shape=sub)
        WORKLOADS["_sample"] = wsub
        model, cfg, w = make_scene("_sample", "cpu")
        sample_n = model.particle_count
    from oracle import oracle as O2

    x = model.particle_q.numpy()
    v = model.particle_qd.numpy()
    consts = cfg.constants(w["dt"], model.particle_max_velocity)
    dims = cfg.resolved_grid_dims()
    a = dict(mass=model.particle_mass.numpy(), inv_mass=model.particle_inv_mass.numpy(),
             flags=model.particle_flags.numpy(), world=model.particle_world.numpy(), gravity=model.gravity.numpy())
    f = np.zeros_like(x)

    def step(x, v):
        r = O2.sph_step(consts, dims, x, v, a["mass"], a["inv_mass"], a["flags"], a["world"], a["gravity"], f_ext=f,
                        v_out_init=v, precision="f32")
        return r["x"], r["v"]

    for _ in range(args.warmup):
        x, v = step(x, v)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        x, v = step(x, v)
    el = time.perf_counter() - t0
    value = sample_n * args.steps / el
    sample = (f"{args.steps} steps of the {sample_n}-particle "
              + (f"{sub[0]}x{sub[1]}x{sub[2]} sub-block of the workload (same spacing and physics)" if sub
                 else "full workload"))
    metric = WORKLOADS[name].get("metric", METRIC)
    line = {
        "impl": "reference",
        "metric": metric,
        "value": value,
        "unit": metric,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": name, "particles": n, "desc": WORKLOADS[name]["desc"]},
        "cpu_baseline": {"value": value, "unit": metric, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def graph_replayed(step):
    """step(a, b) captured into a CUDA graph per (a, b) buffer pair on its
    first use (run eagerly that time), replayed afterwards: how a user
    replays SolverSPH.step with torch.cuda.graph."""
    import torch

    graphs = {}

    def run(a, b):
        key = (a.particle_q.data_ptr(), a.particle_qd.data_ptr(), b.particle_q.data_ptr(), b.particle_qd.data_ptr())
        g = graphs.get(key)
        if g is None:
            step(a, b)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=torch.cuda.current_stream()):
                step(a, b)
            graphs[key] = g
            return
        g.replay()

    run.graphs = graphs
    return run


def pipelined_e2e(model, step, hx, hv, steps: int, device, outputs=None, nbuf: int = 3, copies: bool = True) -> float:
    """Milliseconds for `steps` end-to-end steps through the public API:
    upload (x, v) from the pinned host tensors hx, hv, step(state_in,
    state_out), download outputs(state_out) (default: x, v) into pinned host
    tensors. Three streams (upload, compute, download) and `nbuf` device
    state pairs let the uploads of the next steps and the downloads of the
    previous ones run while a step computes; events order every reuse of a
    buffer. Three pairs: with two, a step k waits for the download of step
    k - 2, and when a step and a copy take about as long (about 0.52 ms each
    on tank_1m) the graph-replayed pipeline fell to 1.70-1.82e9 against
    1.96e9 with three or four pairs (same box, both bounds at 2.0e9).
    Timed with CUDA events from a common start to the last download.
    With copies=False the uploads and downloads are left out (the inputs are
    uploaded once, before the timing): the compute-only bound of the same
    schedule."""
    import torch

    if outputs is None:
        outputs = lambda st: (st.particle_q, st.particle_qd)  # noqa: E731
    s_in, s_c, s_out = (torch.cuda.Stream(device) for _ in range(3))
    ins = [model.state() for _ in range(nbuf)]
    outs = [model.state() for _ in range(nbuf)]
    host_out = [[torch.empty(t.shape, dtype=t.dtype).pin_memory() for t in outputs(outs[b])] for b in range(nbuf)]
    up = [torch.cuda.Event() for _ in range(nbuf)]
    done = [torch.cuda.Event() for _ in range(nbuf)]
    down = [torch.cuda.Event() for _ in range(nbuf)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(device)
    # one untimed round (each buffer once) to warm the streams' first launches
    for k in range(steps + nbuf):
        b = k % nbuf
        if k == nbuf:
            torch.cuda.synchronize()
            start.record(cur)
            for st in (s_in, s_c, s_out):
                st.wait_event(start)
        with torch.cuda.stream(s_in):
            if k >= nbuf:
                s_in.wait_event(done[b])  # step k - nbuf no longer reads ins[b]
            if copies or k < nbuf:
                ins[b].particle_q.copy_(hx, non_blocking=True)
                ins[b].particle_qd.copy_(hv, non_blocking=True)
            up[b].record(s_in)
        with torch.cuda.stream(s_c):
            s_c.wait_event(up[b])
            if k >= nbuf:
                s_c.wait_event(down[b])  # the download of step k - nbuf has read outs[b]
            step(ins[b], outs[b])
            done[b].record(s_c)
        with torch.cuda.stream(s_out):
            s_out.wait_event(done[b])
            if copies:
                for h, t in zip(host_out[b], outputs(outs[b])):
                    h.copy_(t, non_blocking=True)
            down[b].record(s_out)
    end.record(s_out)
    end.synchronize()
    return start.elapsed_time(end)

def load_kernel_counts(kernel: str, workload: str) -> dict:
    """ncu figures of a kernel (profiles/ncu_traffic.json), only when they
    were captured on this workload (its name starts the entry's `workload`)."""
    p = REPO / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return {}
    try:
        c = dict(json.loads(p.read_text()).get(kernel, {}))
    except (ValueError, OSError):
        return {}
    return c if str(c.get("workload", "")).split(" ")[0] == workload else {}


def load_traffic(kernel: str, workload: str):
    return load_kernel_counts(kernel, workload).get("traffic_bytes_per_launch")


def measure_fp32_peak(device) -> dict:
    """FP32 FMA / warp-instruction issue peak of this GPU (nsph_fp32_peak)."""
    import ctypes

    import torch

    from newton_sph_dev_b200 import _lib

    tf, wi, ms = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    st = _lib.load().nsph_fp32_peak(device.index or 0, 4096, ctypes.byref(tf), ctypes.byref(wi), ctypes.byref(ms),
                                    torch.cuda.current_stream(device).cuda_stream)
    _lib.check(st, "nsph_fp32_peak")
    return {"fp32_tflops": tf.value, "warp_inst_per_s": wi.value, "ms": ms.value}


def issue_roofline(kname: str, t_launch_s: float, n: int, peak: dict, workload: str) -> dict:
    """Issue roofline of a neighbour pass: warp instructions per launch (ncu,
    the same workload) over its CUDA-event duration, against the measured
    warp-instruction issue peak."""
    c = load_kernel_counts(kname, workload)
    wi = c.get("warp_inst_per_launch")
    ti = c.get("thread_inst_per_launch")
    out = {"bound": "issue", "kernel": kname, "unit": "warp inst/s", "peak": peak["warp_inst_per_s"],
           "peak_kind": "measured (nsph_fp32_peak: FFMA chains, 64 warps per SM)",
           "fp32_peak_tflops": peak["fp32_tflops"], "warp_inst_per_launch": wi,
           "thread_inst_per_particle": (ti / n) if ti else None, "simt_efficiency": (ti / wi / 32.0) if ti and wi else None,
           "source": c.get("source")}
    if wi:
        out["achieved"] = wi / t_launch_s
        out["frac"] = out["achieved"] / peak["warp_inst_per_s"]
    else:
        out["achieved"] = out["frac"] = None
    return out


def load_peak():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (ValueError, KeyError, OSError):
            pass
    return 6650.0, "fallback"


def run_gpu(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", device_id=device, timeout=timedelta(seconds=120))

    from newton_sph_dev_b200.solvers import SolverSPH

    model, cfg, w = make_scene(args.workload, str(device), rank, world)
    n = model.particle_count
    sharded = "worlds" in w and world > 1  # the worlds are split over the ranks, not replicated
    n_job = sum(world_sizes(worlds_layout(w))) if sharded else world * n
    solver = SolverSPH(model, cfg)
    dt = w["dt"]
    s0, s1 = model.state(), model.state()
    stream = torch.cuda.current_stream(device)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    # the library records start / built / density / end events inside every
    # step (as external event nodes when captured), on the launching stream
    tuned = solver.autotune(s0, s1, dt) if not args.no_autotune else None
    solver.enable_phase_timing(True)

    def step(a, b):
        solver.step(a, b, None, None, dt)

    # warm-up (eager), then capture one graph per ping-pong direction
    for i in range(max(args.warmup, 3)):
        step(s0, s1) if i % 2 == 0 else step(s1, s0)
    torch.cuda.synchronize()
    launches_per_step = solver.last_launches
    use_graph = not args.no_graph
    graphs = None
    if use_graph:
        try:
            ga, gb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
            with torch.cuda.graph(ga):
                step(s0, s1)
            with torch.cuda.graph(gb):
                step(s1, s0)
            graphs = (ga, gb)
            for g in graphs:  # one replay each to validate event timing through graphs
                g.replay()
                solver.phase_times()
        except Exception as exc:  # timing events through graphs unavailable: fall back to eager steps
            print(f"[bench] graph capture unavailable ({exc}); timing eager steps", file=sys.stderr)
            graphs = None
            use_graph = False
            torch.cuda.synchronize()

    # relaxation: the jittered lattice settles over its first ~100 steps, and
    # the timed steps run on the settled state (untimed, an even count so
    # the ping-pong order is unchanged)
    relax = args.relax + (args.relax % 2)
    for i in range(relax):
        if graphs is not None:
            graphs[i % 2].replay()
        else:
            step(s0, s1) if i % 2 == 0 else step(s1, s0)
    torch.cuda.synchronize()

    phase = {"build": 0.0, "density": 0.0, "force": 0.0}
    total_ms = 0.0
    barrier(device)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            if graphs is not None:
                graphs[i % 2].replay()
            else:
                step(s0, s1) if i % 2 == 0 else step(s1, s0)
            t_build, t_dens, t_force = solver.phase_times()
            phase["build"] += t_build
            phase["density"] += t_dens
            phase["force"] += t_force
            total_ms += t_build + t_dens + t_force
    torch.cuda.synchronize()
    barrier(device)
    total_ms_max = max_over_ranks(total_ms, device)
    status = solver.status()
    timed_state = s1 if args.steps % 2 == 1 else s0  # the last timed step's output

    value = n_job * args.steps / (total_ms_max * 1e-3)
    ms_per_step = total_ms_max / args.steps

    # ---- end to end through the public API with host buffers ----
    e2e_steps = min(args.steps, 100)
    # the host copy of the timed run's last state (not the initial lattice)
    hx = timed_state.particle_q.cpu().pin_memory()
    hv = timed_state.particle_qd.cpu().pin_memory()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # a solver as a user makes it: the timed run's launch shape, without the
    # phase events the timed run records inside every step
    user_solver = SolverSPH(model, cfg)
    if hasattr(solver, "launch"):
        user_solver.set_launch(*solver.launch)
    # (a) pipelined: every step uploads its inputs from pinned host memory,
    # runs SolverSPH.step and downloads its result; the upload of step k+1
    # and the download of step k-1 overlap the step k on their own streams
    barrier(device)
    torch.cuda.synchronize()
    # each step replays SolverSPH.step captured with torch.cuda.graph (the
    # first use of each buffer pair, in the untimed warm-up round, captures)
    gstep = graph_replayed(lambda a, b: user_solver.step(a, b, None, None, dt))
    e2e_ms = pipelined_e2e(model, gstep, hx, hv, e2e_steps, device)
    barrier(device)
    e2e_ms_max = max_over_ranks(e2e_ms, device)
    e2e_value = n_job * e2e_steps / (e2e_ms_max * 1e-3)
    # the same schedule and graphs with no uploads or downloads: the compute's
    # bound on (a) (no L2 flush between these steps, unlike the timed run)
    barrier(device)
    torch.cuda.synchronize()
    step_ms = max_over_ranks(pipelined_e2e(model, gstep, hx, hv, e2e_steps, device, copies=False), device)
    e2e_step_bound = n_job * e2e_steps / (step_ms * 1e-3)
    gstep.graphs.clear()
    # the same with eager SolverSPH.step calls
    barrier(device)
    torch.cuda.synchronize()
    eager_ms = max_over_ranks(pipelined_e2e(model, lambda a, b: user_solver.step(a, b, None, None, dt), hx, hv,
                                            e2e_steps, device), device)
    e2e_eager = n_job * e2e_steps / (eager_ms * 1e-3)
    # the same uploads and downloads with no step between them: the host
    # link's bound on (a)
    barrier(device)
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(pipelined_e2e(model, lambda a, b: None, hx, hv, e2e_steps, device), device)
    e2e_copy_bound = n_job * e2e_steps / (copy_ms * 1e-3)
    # (b) serial host round trip: upload, step, download, and the next step
    # starts from the downloaded state
    serial_ms = 0.0
    torch.cuda.synchronize()
    for _ in range(e2e_steps):
        e0.record(stream)
        s0.particle_q.copy_(hx, non_blocking=True)
        s0.particle_qd.copy_(hv, non_blocking=True)
        user_solver.step(s0, s1, None, None, dt)
        hx.copy_(s1.particle_q, non_blocking=True)
        hv.copy_(s1.particle_qd, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        serial_ms += e0.elapsed_time(e1)
    del user_solver
    barrier(device)
    serial_ms = max_over_ranks(serial_ms, device)
    e2e_serial = world * n * e2e_steps / (serial_ms * 1e-3)
    state_bytes = n * 3 * 4 * 2

    # ---- roofline of the dominant single-kernel pass ----
    peak, peak_kind = load_peak()
    dom = "force" if phase["force"] >= phase["density"] else "density"
    b_alg = (B_ALG_FORCE if dom == "force" else B_ALG_DENSITY) * n
    t_launch = phase[dom] / args.steps * 1e-3
    achieved = b_alg / t_launch / 1e9
    kname = "k_force_list" if dom == "force" else "k_density_list"
    traffic = load_traffic(kname, args.workload)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "alg_bytes_per_launch": b_alg}
    step_achieved = B_ALG_STEP * n / (ms_per_step * 1e-3) / 1e9
    roofline_step = {"bound": "hbm", "achieved": step_achieved, "peak": peak, "unit": "GB/s",
                     "frac": step_achieved / peak, "alg_bytes_per_particle_step": B_ALG_STEP}

    fp32 = measure_fp32_peak(device)
    roof_issue = issue_roofline(kname, t_launch, n, fp32, args.workload)

    # the same timed steps in the tolerance arithmetic (graph-replayed, L2
    # flushed, from the timed state); the headline stays the exact arithmetic
    fast = None
    if not isinstance(cfg, list) and use_graph:
        solver.set_arithmetic("fast")
        fa, fb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        step(s0, s1)
        with torch.cuda.graph(fa):
            step(s0, s1)
        with torch.cuda.graph(fb):
            step(s1, s0)
        fph = {"build": 0.0, "density": 0.0, "force": 0.0}
        for i in range(args.steps):
            flush.zero_()
            (fa if i % 2 == 0 else fb).replay()
            tb, td, tf = solver.phase_times()
            fph["build"] += tb
            fph["density"] += td
            fph["force"] += tf
        fms = sum(fph.values())
        del fa, fb
        solver.set_arithmetic("exact")
        fast = {"value": n * args.steps / (fms * 1e-3), "ms_per_step": fms / args.steps,
                "phase_ms_per_step": {k: v / args.steps for k, v in fph.items()},
                "arithmetic": "hardware rsqrt in the kernel terms; same neighbour sets and summation order; "
                              "parity against the fp64 oracle (tests/test_gpu_fullsize.py)"}

    # the learned surrogate beside the plain step, from the timed state (the
    # three arms of surrogate_eval; not part of the headline value)
    surrogate = surrogate_8x = None
    if not isinstance(cfg, list) and args.surrogate_calls > 0:
        surrogate = surrogate_eval(solver, model, 4, dt, args.surrogate_calls, timed_state.particle_q.clone(),
                                   timed_state.particle_qd.clone(), device)
        if args.workload.startswith("tank_"):  # dt = 5e-5: one step of 4e-4 s = 8 plain steps
            from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel

            sw8 = WORKLOADS["tank_1m_surrogate_8x"]["surrogate"]
            net8 = SurrogateModel.load(REPO / "newton_sph_dev_b200" / sw8["weights"], device)
            surrogate_8x = surrogate_eval(solver, model, sw8["substeps"], dt, args.surrogate_calls,
                                          timed_state.particle_q.clone(), timed_state.particle_qd.clone(), device,
                                          net=net8, threshold=sw8["threshold"], window=sw8["window"])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model_cpu, cfg_cpu, w_cpu = make_scene(args.workload, "cpu")
        if isinstance(cfg_cpu, list):
            rate, nw, el, threads = cpu_oracle_rate(model_cpu, cfg_cpu, w_cpu, budget_s=15.0, max_steps=len(cfg_cpu))
            sample = f"one step of each of the first {nw} worlds in {el:.1f} s (fp32 oracle, OpenMP)"
        else:
            rate, steps_done, el, threads = cpu_oracle_rate(model_cpu, cfg_cpu, w_cpu, budget_s=15.0, max_steps=40)
            sample = f"{steps_done} full steps of the {n}-particle workload in {el:.1f} s (fp32 oracle, OpenMP)"
        cpu = {"value": rate, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample}

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC,
            "value": value,
            "unit": METRIC,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "strong" if sharded else "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": args.workload,
                "particles": n_job if sharded else n,
                "desc": w["desc"],
                "grid_dims": list(solver.grid_dims) if solver.grid_dims is not None else "per world (tight)",
                "worlds": w["worlds"] if sharded else model.world_count,
                "graph": use_graph,
                "launch": {"threads": solver.launch[0], "blocks_per_sm": solver.launch[1],
                           "autotuned": tuned is not None} if hasattr(solver, "launch") else "default",
                "l2": "flushed (256 MiB write) before every timed step, outside the timed interval",
                "relaxation_steps": relax,
                "parallelism": (f"worlds split over {world} GPUs by particle count (rank 0: {model.world_count} "
                                f"worlds, {n} particles); no collective in the step" if sharded
                                else f"replicas x{world}" if world > 1 else "single GPU"),
            },
            "phase_ms_per_step": {k: v / args.steps for k, v in phase.items()},
            "roofline": roofline,
            "roofline_step": roofline_step,
            "roofline_issue": roof_issue,
            "fast_arithmetic": fast,
            "surrogate": surrogate,
            "surrogate_8x": surrogate_8x,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": e2e_steps,
                    "how": "each step uploads x, v from pinned host memory, runs SolverSPH.step (captured with "
                           "torch.cuda.graph, replayed) and downloads x, v; independent steps from the same host "
                           "state (the timed run's last state), uploads and downloads overlapping other steps' "
                           "compute on separate streams (three device state pairs); a second SolverSPH on the "
                           "same model with the timed run's launch shape and no phase-timing events",
                    "eager": {"value": e2e_eager, "how": "the same with eager SolverSPH.step calls"},
                    "copy_bound": {"value": e2e_copy_bound,
                                   "how": "the same uploads and downloads with no step between them (the host "
                                          "link's bound on the pipelined figure)"},
                    "step_bound": {"value": e2e_step_bound,
                                   "how": "the same graph-replayed steps with no uploads or downloads (the "
                                          "compute's bound on the pipelined figure; unlike the timed run, no L2 "
                                          "flush between steps and no phase-timing events)"},
                    "serial_round_trip": {"value": e2e_serial, "how": "upload, eager step, download, next step "
                                                                      "from the downloaded state, no overlap"}},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "status": status,
        }
        print(json.dumps(line), flush=True)
    if graphs is not None:
        del graphs
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# differentiable rollout (adjoint): forward + checkpointed backward
# ---------------------------------------------------------------------------
# algorithmic bytes per particle of the pair gather of the adjoint (read x, v,
# the density-pass scratch, adj(a), adj(dv); read-modify-write adj(x), adj(v);
# write adj(rho))
B_ALG_ADJ_PAIR = 16 + 16 + 8 + 8 + 16 + 16 + 24 + 24 + 4


def grad_target(x: np.ndarray, w: dict) -> np.ndarray:
    """The seeded target cloud of the differentiable-rollout workload: the
    initial block shifted by (s, 0, -s/2) plus N(0, (0.2 s)^2) noise."""
    s = w["spacing"]
    rng = np.random.default_rng(w["grad"]["target_seed"])
    return (x + np.array([s, 0.0, -0.5 * s]) + rng.normal(0.0, 0.2 * s, x.shape)).astype(np.float32)


def cpu_grad_rate(model_cpu, cfg, w, budget_s: float):
    """Differentiable particle-steps/s of the fp64 adjoint oracle (forward
    passes on all OpenMP threads, reverse pass on one thread) over a bounded
    number of steps of the same scene."""
    from oracle import oracle as O

    O.build()
    x = model_cpu.particle_q.numpy().astype(np.float64)
    v = model_cpu.particle_qd.numpy().astype(np.float64)
    y = grad_target(model_cpu.particle_q.numpy(), w)
    sc = O.AdjScene(cfg.constants(w["dt"], model_cpu.particle_max_velocity)["f64"], model_cpu.particle_mass.numpy(),
                    model_cpu.particle_inv_mass.numpy(), model_cpu.particle_flags.numpy(),
                    model_cpu.gravity.numpy())
    t0 = time.perf_counter()
    O.rollout_grad64(sc, x, v, 1, y)
    per_step = time.perf_counter() - t0
    steps = int(max(1, min(w["grad"]["steps"], budget_s / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    O.rollout_grad64(sc, x, v, steps, y)
    el = time.perf_counter() - t0
    n = x.shape[0]
    return n * steps / el, steps, el, O.get_threads()


def run_grad(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", device_id=device, timeout=timedelta(seconds=120))
    from newton_sph_dev_b200.solvers import SolverSPH, sph_rollout

    model, cfg, w = make_scene(args.workload, str(device))
    n = model.particle_count
    g = w["grad"]
    steps, every, dt = g["steps"], g["checkpoint"], w["dt"]
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    tuned = solver.autotune(s0, s1, dt) if not args.no_autotune else None
    solver.enable_adjoint()
    solver.enable_phase_timing(True)
    x0d = model.particle_q.clone()
    v0d = model.particle_qd.clone()
    y = torch.from_numpy(grad_target(model.particle_q.cpu().numpy(), w)).to(device)
    b0 = torch.tensor([float(solver.step_params(dt).eos_b)], dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def rollout(x0, v0, b, timed):
        if timed:
            ev[0].record(stream)
        xT, _ = sph_rollout(solver, x0, v0, steps, dt, eos_b=b, checkpoint_every=every)
        loss = ((xT - y) ** 2).sum(dim=1).mean()
        if timed:
            ev[1].record(stream)
        loss.backward()
        if timed:
            ev[2].record(stream)
        return loss

    def leaves():
        return (x0d.detach().clone().requires_grad_(True), v0d.detach().clone().requires_grad_(True),
                b0.detach().clone().requires_grad_(True))

    for _ in range(args.warmup):
        rollout(*leaves(), timed=False)
    torch.cuda.synchronize()
    fwd_ms = bwd_ms = 0.0
    dens_ms = pair_ms = 0.0
    launches0 = solver.launches_total
    barrier(device)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            x0, v0, b = leaves()
            flush.zero_()
            loss = rollout(x0, v0, b, timed=True)
            ev[2].synchronize()
            fwd_ms += ev[0].elapsed_time(ev[1])
            bwd_ms += ev[1].elapsed_time(ev[2])
            ph = solver.adjoint_phase_times()  # the last adjoint step of this rollout
            dens_ms += solver.phase_times()[1]  # the last forward step's density pass
            pair_ms += ph[3]
    torch.cuda.synchronize()
    barrier(device)
    launches = solver.launches_total - launches0
    total_ms = max_over_ranks(fwd_ms + bwd_ms, device)
    value = world * n * steps * args.steps / (total_ms * 1e-3)
    grads_finite = bool(torch.isfinite(x0.grad).all() and torch.isfinite(v0.grad).all() and torch.isfinite(b.grad).all())

    # ---- end to end through the public API, host buffers in and out ----
    e2e_iters = min(args.steps, 20)
    hx, hv = x0d.cpu().pin_memory(), v0d.cpu().pin_memory()
    hgx, hgv = torch.empty_like(hx).pin_memory(), torch.empty_like(hv).pin_memory()
    hb = torch.empty(2, dtype=torch.float32).pin_memory()
    e2e_ms = 0.0
    barrier(device)
    torch.cuda.synchronize()
    for _ in range(e2e_iters):
        ev[0].record(stream)
        x0 = hx.to(device, non_blocking=True).requires_grad_(True)
        v0 = hv.to(device, non_blocking=True).requires_grad_(True)
        b = b0.detach().clone().requires_grad_(True)
        loss = rollout(x0, v0, b, timed=False)
        hgx.copy_(x0.grad, non_blocking=True)
        hgv.copy_(v0.grad, non_blocking=True)
        hb[0:1].copy_(loss.detach().reshape(1), non_blocking=True)
        hb[1:2].copy_(b.grad, non_blocking=True)
        ev[2].record(stream)
        ev[2].synchronize()
        e2e_ms += ev[0].elapsed_time(ev[2])
    barrier(device)
    e2e_ms = max_over_ranks(e2e_ms, device)
    e2e_value = world * n * steps * e2e_iters / (e2e_ms * 1e-3)

    # ---- roofline: the density pass has the largest share of the rollout's
    # kernel time (it runs in the forward and the segment recompute steps); the
    # pair gather is the adjoint's largest single kernel ----
    peak, peak_kind = load_peak()
    t_dens = dens_ms / args.steps * 1e-3
    t_pair = pair_ms / args.steps * 1e-3
    achieved = B_ALG_DENSITY * n / t_dens / 1e9
    roofline = {"bound": "hbm", "kernel": "k_density_list", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                "alg_bytes_per_launch": B_ALG_DENSITY * n}
    pair_ach = B_ALG_ADJ_PAIR * n / t_pair / 1e9
    roofline_adj = {"bound": "hbm", "kernel": "k_adj_pair", "achieved": pair_ach, "peak": peak, "unit": "GB/s",
                    "frac": pair_ach / peak, "alg_bytes_per_launch": B_ALG_ADJ_PAIR * n,
                    "ms_per_launch": t_pair * 1e3}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model_cpu, cfg_cpu, w_cpu = make_scene(args.workload, "cpu")
        rate, csteps, el, threads = cpu_grad_rate(model_cpu, cfg_cpu, w_cpu, budget_s=15.0)
        cpu = {"value": rate, "unit": "differentiable particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"forward + reverse of {csteps} steps of the full {n}-particle scene in {el:.1f} s "
                         f"(fp64 adjoint oracle: forward passes on {threads} OpenMP threads, reverse pass on one)"}

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": "differentiable particle-steps/s",
            "value": value,
            "unit": "differentiable particle-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": args.workload,
                "particles": n,
                "desc": w["desc"],
                "step": "one bench step = one forward rollout + loss + checkpointed backward "
                        f"({steps} simulation steps); value counts particle x simulation steps",
                "grid_dims": list(solver.grid_dims),
                "launch": {"threads": solver.launch[0], "blocks_per_sm": solver.launch[1],
                           "autotuned": tuned is not None} if hasattr(solver, "launch") else "default",
                "l2": "flushed (256 MiB write) before every timed rollout, outside the timed interval",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "phase_ms_per_step": {"forward": fwd_ms / args.steps, "backward": bwd_ms / args.steps},
            "roofline": roofline,
            "roofline_adjoint_pair": roofline_adj,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "differentiable particle-steps/s",
                    "h2d_bytes_per_step": 2 * n * 12, "d2h_bytes_per_step": 2 * n * 12 + 8, "steps": e2e_iters},
            "gpu_launches": launches,
            "clocks": clocks,
            "grads_finite": grads_finite,
            "loss": float(loss.item()),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_grad_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    model, cfg, w = make_scene(args.workload, "cpu")
    n = model.particle_count
    from oracle import oracle as O

    O.build()
    x = model.particle_q.numpy().astype(np.float64)
    v = model.particle_qd.numpy().astype(np.float64)
    y = grad_target(model.particle_q.numpy(), w)
    sc = O.AdjScene(cfg.constants(w["dt"], model.particle_max_velocity)["f64"], model.particle_mass.numpy(),
                    model.particle_inv_mass.numpy(), model.particle_flags.numpy(), model.gravity.numpy())
    t0 = time.perf_counter()
    O.rollout_grad64(sc, x, v, 1, y)
    per_step = time.perf_counter() - t0
    # each bench step: forward + reverse of a bounded number of simulation steps
    budget = 150.0 / (args.steps + args.warmup)
    sim_steps = int(max(1, min(w["grad"]["steps"], budget / max(per_step, 1e-6))))
    for _ in range(args.warmup):
        O.rollout_grad64(sc, x, v, sim_steps, y)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.rollout_grad64(sc, x, v, sim_steps, y)
    el = time.perf_counter() - t0
    value = n * sim_steps * args.steps / el
    unit = "differentiable particle-steps/s"
    threads = O.get_threads()
    line = {
        "impl": "reference", "metric": unit, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "desc": w["desc"]},
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                         "sample": f"each step: forward + reverse of {sim_steps} simulation steps of the full scene "
                                   f"(fp64 adjoint oracle; forward passes on {threads} OpenMP threads, reverse on "
                                   f"one)"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# learned surrogate step (4 x dt per step, plain step as fallback and yardstick)
# ---------------------------------------------------------------------------
# algorithmic bytes per particle: feature pass (read x, v, m/rho p/rho^2, rho p;
# write 16 features, a, dv) and MLP + integrate (read them back with x, v,
# rho p and the sort permutation; write x, v)
# algorithmic bytes per particle of the fused surrogate kernel: read x, v (sorted mirrors, 32), the density
# scratch (16), the neighbour-list count (4); write x, v (24)
B_ALG_FUSED = 32 + 16 + 4 + 24
MLP_FLOPS = 2 * (16 * 64 + 64 * 64 + 64 * 16)  # per particle, as issued (layer 3 padded to N = 16)


def load_tensor_peak():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
        except (ValueError, KeyError, OSError):
            pass
    return 1590.0, "fallback"


def surrogate_eval(solver, model, sub: int, dt: float, calls: int, start_q, start_qd, device, net=None,
                   threshold: float = 0.01, window: int = 10, phase_timing: bool = True) -> dict:
    """Three arms from the same state, each over the same span of simulated
    time (calls x sub x dt), each call replayed from a CUDA graph with L2
    flushed before it:

    - surrogate: SurrogateSPH (one corrected step of sub x dt per call, plain
      fallback under the compression rule);
    - uncorrected: the same large step with a zero network (the plain WCSPH
      step at sub x dt), no fallback;
    - plain: sub x calls plain steps of dt.

    Rates are particles x plain-dt steps of simulated time per second."""
    import torch

    from newton_sph_dev_b200.solvers.sph_surrogate import SurrogateModel, SurrogateSPH

    n = model.particle_count
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"calls": calls, "substeps": sub, "dt_plain": dt, "dt_large": sub * dt}

    def arm(network, thr):
        a, b = model.state(), model.state()
        a.particle_q.copy_(start_q)
        a.particle_qd.copy_(start_qd)
        st = SurrogateSPH(solver, network, substeps=sub, threshold=thr, window=window, graphs=True)
        # capture both ping-pong directions with two untimed calls, then start over
        st.step(a, b, dt)
        st.step(b, a, dt)
        a.particle_q.copy_(start_q)
        a.particle_qd.copy_(start_qd)
        st.reset_counters()
        solver.reset_status()
        ms = fused_ms = 0.0
        cur, nxt = a, b
        diverged_at = None
        done = 0
        torch.cuda.synchronize()
        by_kind = {"surrogate": 0.0, "plain": 0.0, "rollback": 0.0}
        for c in range(calls):
            flush.zero_()
            before = st.surrogate_steps
            rb = st.rollbacks
            e0.record(stream)
            st.step(cur, nxt, dt)
            e1.record(stream)
            e1.synchronize()
            t_call = e0.elapsed_time(e1)
            ms += t_call
            by_kind["rollback" if st.rollbacks > rb else ("surrogate" if st.surrogate_steps > before else "plain")] += t_call
            if phase_timing and st.surrogate_steps > before:
                fused_ms += solver.surrogate_phase_times()[2]
            cur, nxt = nxt, cur
            done += 1
            # an arm whose state has blown up is stopped (its neighbour
            # counts explode and each further call only gets slower)
            if (c + 1) % window == 0 and not bool(torch.isfinite(cur.particle_q).all()):
                diverged_at = c + 1
                break
        finite = bool(torch.isfinite(cur.particle_q).all() and torch.isfinite(cur.particle_qd).all())
        res = {"value": n * sub * done / (ms * 1e-3), "ms_per_call": ms / done, "calls_run": done,
               "diverged_at_call": diverged_at,
               "mean_compression": st.mean_compression(),
               "max_window_compression": st.committed_window_worst(),
               "surrogate_steps": st.surrogate_steps, "fallback_calls": st.fallback_calls,
               "rollbacks": st.rollbacks, "rejected_window_worst": float(max(st.rejected_worst or [0.0])),
               "timeouts": st.timeouts, "finite": finite, "status": solver.status(),
               "ms_by_call_kind": by_kind,
               "fused_kernel_ms": fused_ms / max(1, st.surrogate_steps) if phase_timing else None,
               "launches_per_call": st.launches_per_step}
        st._graphs.clear()
        return res

    net = net if net is not None else SurrogateModel.pretrained(device)
    out["surrogate"] = arm(net, threshold)
    zero = SurrogateModel(device)
    zero.zero_correction()
    out["uncorrected"] = arm(zero, float("inf"))

    # plain: sub x calls steps of dt from the same state
    p0, p1 = model.state(), model.state()
    for t in (p0, p1):
        t.particle_q.copy_(start_q)
        t.particle_qd.copy_(start_qd)
    solver.step(p0, p1, None, None, dt)
    ga, gb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(ga):
        solver.step(p0, p1, None, None, dt)
    with torch.cuda.graph(gb):
        solver.step(p1, p0, None, None, dt)
    p0.particle_q.copy_(start_q)
    p0.particle_qd.copy_(start_qd)
    plain_ms = 0.0
    torch.cuda.synchronize()
    for i in range(sub * calls):
        flush.zero_()
        e0.record(stream)
        (ga if i % 2 == 0 else gb).replay()
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
    del ga, gb
    out["plain"] = {"value": n * sub * calls / (plain_ms * 1e-3), "ms_per_step": plain_ms / (sub * calls)}
    out["speedup_vs_plain"] = out["surrogate"]["value"] / out["plain"]["value"]
    out["speedup_vs_uncorrected"] = out["surrogate"]["value"] / out["uncorrected"]["value"]
    out["compression_definition"] = "mean over active particles of max(0, rho/rho0 - 1) at each large step's input"
    return out


def run_surrogate(args):
    """The learned surrogate on the tank: the three arms of surrogate_eval
    (surrogate, uncorrected large step, plain steps) over args.steps calls
    from the relaxed state; the headline value is the surrogate's."""
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", device_id=device, timeout=timedelta(seconds=120))
    from newton_sph_dev_b200.solvers import SolverSPH
    from newton_sph_dev_b200.solvers.sph_surrogate import FallbackMonitor, SurrogateModel, SurrogateSPH

    model, cfg, w = make_scene(args.workload, str(device))
    n = model.particle_count
    sw = w["surrogate"]
    sub, dt = sw["substeps"], w["dt"]
    solver = SolverSPH(model, cfg)
    s0, s1 = model.state(), model.state()
    tuned = solver.autotune(s0, s1, dt) if not args.no_autotune else None
    solver.enable_phase_timing(True)
    # relaxation with plain steps, then every arm starts from that state
    relax = max(args.warmup, 3) + args.relax
    relax += relax % 2
    for i in range(relax):
        solver.step(s0, s1, None, None, dt) if i % 2 == 0 else solver.step(s1, s0, None, None, dt)
    torch.cuda.synchronize()
    start_q, start_qd = s0.particle_q.clone(), s0.particle_qd.clone()
    weights = args.weights or sw.get("weights")
    if weights:
        path = Path(weights)
        if not path.is_absolute() and not path.exists():
            path = REPO / "newton_sph_dev_b200" / weights
        net = SurrogateModel.load(path, device)
    else:
        net = SurrogateModel.pretrained(device)
    barrier(device)
    with ClockSampler(local) as clk:
        ev = surrogate_eval(solver, model, sub, dt, args.steps, start_q, start_qd, device, net=net,
                            threshold=sw["threshold"], window=sw["window"])
    sur = ev["surrogate"]
    total_ms = max_over_ranks(sur["ms_per_call"] * args.steps, device)
    value = world * n * sub * args.steps / (total_ms * 1e-3)
    status = sur["status"]  # the surrogate arm's (the uncorrected arm may blow up by design)

    # end to end through the public API: host state in, one call, host state
    # out, every call (pipelined over independent calls, as for tank_1m), all
    # from the relaxed state with the fallback rule reset
    e2e_steps = min(args.steps, 50)
    hx, hv = start_q.cpu().pin_memory(), start_qd.cpu().pin_memory()
    # a solver as a user makes it: the same launch shape, no phase-timing events
    user_solver = SolverSPH(model, cfg)
    user_solver.set_launch(*solver.launch)
    stepper = SurrogateSPH(user_solver, net, substeps=sub, threshold=sw["threshold"], window=sw["window"],
                           graphs=True)
    stepper.monitor = FallbackMonitor(sw["threshold"])
    e2e_ms = pipelined_e2e(model, lambda a, b: stepper.step(a, b, dt), hx, hv, e2e_steps, device)
    e2e_ms = max_over_ranks(e2e_ms, device)
    e2e_value = world * n * sub * e2e_steps / (e2e_ms * 1e-3)
    e2e_fallbacks = stepper.fallback_calls
    stepper._graphs.clear()
    del stepper, user_solver

    peak, peak_kind = load_peak()
    tpeak, tpeak_kind = load_tensor_peak()
    t_fused = (sur["fused_kernel_ms"] or 0.0) * 1e-3
    ach = B_ALG_FUSED * n / t_fused / 1e9 if t_fused > 0 else None
    roofline = {"bound": "hbm", "kernel": "k_surrogate_fused (features + MLP + integrate)", "achieved": ach,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": ach / peak if ach else None,
                "traffic": load_traffic("k_surrogate_fused", args.workload), "alg_bytes_per_launch": B_ALG_FUSED * n,
                "ms_per_launch": t_fused * 1e3}
    tflops = MLP_FLOPS * n / t_fused / 1e12 if t_fused > 0 else None
    roofline_mlp = {"bound": "tensor", "kernel": "k_surrogate_fused (its MLP share)", "achieved": tflops,
                    "peak": tpeak, "peak_kind": tpeak_kind, "unit": "TFLOP/s",
                    "frac": tflops / tpeak if tflops else None, "flops_per_particle": MLP_FLOPS,
                    "note": "MLP flops as issued over the fused kernel's whole duration (the neighbour gather "
                            "dominates it)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model_cpu, cfg_cpu, w_cpu = make_scene(args.workload, "cpu")
        rate, steps_done, el, threads = cpu_oracle_rate(model_cpu, cfg_cpu, w_cpu, budget_s=15.0, max_steps=40)
        cpu = {"value": rate, "unit": w["metric"], "cores": threads, "kind": "port",
               "sample": f"{steps_done} plain fp32 oracle steps (dt = {dt} s) of the full {n}-particle scene in "
                         f"{el:.1f} s (OpenMP); the CPU has no surrogate, one plain step is one dt of simulated time"}
    if rank == 0:
        line = {
            "metric": w["metric"],
            "value": value,
            "unit": w["metric"],
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (MLP bf16, fp32 accumulate)",
            "data": "synthetic",
            "config": {
                "workload": args.workload, "particles": n, "desc": w["desc"],
                "step": f"one bench step = one call advancing {sub} x {dt} s of simulated time; value counts "
                        f"particles x plain-dt steps of simulated time",
                "substeps": sub, "dt_plain": dt, "dt_surrogate": sub * dt, "fallback_threshold": sw["threshold"],
                "window": sw["window"], "graph": True, "relaxation_steps": relax,
                "launch": {"threads": solver.launch[0], "blocks_per_sm": solver.launch[1],
                           "autotuned": tuned is not None} if hasattr(solver, "launch") else "default",
                "l2": "flushed (256 MiB write) before every timed call, outside the timed interval",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            },
            "arms": ev,
            "speedup_vs_plain": ev["speedup_vs_plain"],
            "speedup_vs_uncorrected": ev["speedup_vs_uncorrected"],
            "compression_error": {"mean": sur["mean_compression"], "max_window": sur["max_window_compression"],
                                  "definition": ev["compression_definition"]},
            "roofline": roofline,
            "roofline_mlp": roofline_mlp,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": w["metric"], "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n,
                    "steps": e2e_steps, "how": "pinned upload, one SurrogateSPH.step call, download, every call; "
                                              "independent calls pipelined on upload / compute / download streams",
                    "state": "the relaxed state, fallback rule reset", "fallback_calls": e2e_fallbacks},
            "gpu_launches": sur["launches_per_call"] * (sur["surrogate_steps"] + sur["rollbacks"] * sw["window"])
            + sur["fallback_calls"] * sub * solver.last_launches,
            "clocks": clk.summary(),
            "status": status,
            "finite": sur["finite"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# particle-particle contact (the reference's semi-implicit contact forces)
# ---------------------------------------------------------------------------
B_ALG_CONTACT = 12 + 12 + 4 + 4 + 12  # read x, v, radius, flags; write f (the sorted mirrors are scratch)


def make_contact_scene(w, device):
    import newton_sph_dev_b200 as nsph
    import torch

    s = w["spacing"]
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(s / 2, s / 2, s / 2), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=w["shape"][0],
                        dim_y=w["shape"][1], dim_z=w["shape"][2], cell_x=s, cell_y=s, cell_z=s, mass=1.0,
                        jitter=0.2 * s, radius_mean=w["radius"])
    model = b.finalize(device)
    rng = np.random.default_rng(seed=2)
    model.particle_qd.copy_(torch.from_numpy(rng.normal(0.0, w["vel_std"], (model.particle_count, 3))
                                             .astype(np.float32)))
    model.particle_cohesion = 0.0
    return model


def run_contact(args):
    import torch

    from newton_sph_dev_b200.contacts import eval_particle_contact_forces

    world, rank, local = dist_env()
    if world > 1:
        raise SystemExit("contact_1m runs on one GPU (replicas are not wired for it)")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    w = WORKLOADS[args.workload]
    model = make_contact_scene(w, str(device))
    n = model.particle_count
    state = model.state()
    f = torch.zeros_like(state.particle_q)
    gr = 2.0 * model.particle_max_radius + model.particle_cohesion
    grid = model.particle_grid
    stream = torch.cuda.current_stream(device)

    def step():
        grid.build(state.particle_q, gr)
        eval_particle_contact_forces(model, state, f)

    for _ in range(max(args.warmup, 3)):
        step()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    total = build_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            ev[0].record(stream)
            grid.build(state.particle_q, gr)
            ev[1].record(stream)
            eval_particle_contact_forces(model, state, f)
            ev[2].record(stream)
            ev[2].synchronize()
            build_ms += ev[0].elapsed_time(ev[1])
            total += ev[0].elapsed_time(ev[2])
    # graph-replayed steps (the same work, one launch sequence)
    gtotal = 0.0
    for _ in range(args.steps):
        flush.zero_()
        ev[0].record(stream)
        g.replay()
        ev[2].record(stream)
        ev[2].synchronize()
        gtotal += ev[0].elapsed_time(ev[2])
    del g
    best = min(total, gtotal)
    value = n * args.steps / (best * 1e-3)
    t_contact = (total - build_ms) / args.steps * 1e-3
    peak, peak_kind = load_peak()
    ach = B_ALG_CONTACT * n / t_contact / 1e9
    roofline = {"bound": "hbm", "kernel": "k_contact_forces", "achieved": ach, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": ach / peak, "traffic": None, "alg_bytes_per_launch": B_ALG_CONTACT * n,
                "ms_per_launch": t_contact * 1e3}
    # end to end: host positions and velocities in, forces out, every step
    # (pipelined over independent steps, as for tank_1m)
    hx, hv = state.particle_q.cpu().pin_memory(), state.particle_qd.cpu().pin_memory()
    e2e_steps = min(args.steps, 50)

    def e2e_step(a, b):
        grid.build(a.particle_q, gr)
        eval_particle_contact_forces(model, a, b.particle_f)

    e2e = pipelined_e2e(model, e2e_step, hx, hv, e2e_steps, device, outputs=lambda st: (st.particle_f,))
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        m = model
        xs, vs = state.particle_q.cpu().numpy(), state.particle_qd.cpu().numpy()
        rr, fl = m.particle_radius.cpu().numpy(), m.particle_flags.cpu().numpy()
        t0 = time.perf_counter()
        reps = 0
        while True:
            O.particle_contact_forces(xs, vs, rr, fl, float(np.float32(gr)), (128, 128, 128), m.particle_ke,
                                      m.particle_kd, m.particle_kf, m.particle_mu, m.particle_cohesion,
                                      m.particle_max_radius)
            reps += 1
            el = time.perf_counter() - t0
            if el > 10.0 or reps >= 20:
                break
        cpu = {"value": n * reps / el, "unit": METRIC, "cores": O.get_threads(), "kind": "port",
               "sample": f"{reps} steps (grid build + contact forces) of the full scene in {el:.1f} s "
                         "(fp32 restatement of eval_particle_contact, OpenMP)"}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": best / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "desc": w["desc"], "grid_dims": [128, 128, 128],
                   "graph": gtotal <= total,
                   "l2": "flushed (256 MiB write) before every timed step, outside the timed interval"},
        "phase_ms_per_step": {"build": build_ms / args.steps, "contact": t_contact * 1e3},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": n * e2e_steps / (e2e * 1e-3), "unit": METRIC, "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 12 * n, "steps": e2e_steps,
                "how": "pinned upload of x, v, grid build + contact forces, download of f, every step; independent "
                       "steps pipelined on upload / compute / download streams"},
        "gpu_launches": (grid.last_launches + 2) * args.steps,  # grid build + mirror gather + contact
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def make_xpbd_scene(w, device):
    import newton_sph_dev_b200 as nsph
    import torch

    s = w["spacing"]
    b = nsph.ModelBuilder()
    b.add_particle_grid(pos=(s / 2, s / 2, w["radius"]), rot=(0, 0, 0, 1), vel=(0, 0, 0), dim_x=w["shape"][0],
                        dim_y=w["shape"][1], dim_z=w["shape"][2], cell_x=s, cell_y=s, cell_z=s, mass=1.0,
                        jitter=0.2 * s, radius_mean=w["radius"])
    b.add_ground_plane()
    model = b.finalize(device)
    rng = np.random.default_rng(seed=2)
    model.particle_qd.copy_(torch.from_numpy(rng.normal(0.0, w["vel_std"], (model.particle_count, 3))
                                             .astype(np.float32)))
    model.particle_cohesion = 0.0
    return model


def run_xpbd(args):
    """SolverXPBD on the sphere pile: Model.collide + step per bench step,
    replayed from a CUDA graph per ping-pong direction."""
    import torch

    from newton_sph_dev_b200.solvers import SolverXPBD

    world, rank, local = dist_env()
    if world > 1:
        raise SystemExit("xpbd_1m runs on one GPU (replicas are not wired for it)")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    w = WORKLOADS[args.workload]
    model = make_xpbd_scene(w, str(device))
    n = model.particle_count
    it, dt = w["xpbd"]["iterations"], w["xpbd"]["dt"]
    solver = SolverXPBD(model, iterations=it)
    s0, s1 = model.state(), model.state()
    contacts = model.contacts()
    stream = torch.cuda.current_stream(device)

    def step(a, b):
        model.collide(a, contacts)
        solver.step(a, b, None, contacts, dt)

    for i in range(max(args.warmup, 3) + args.relax // 10):
        step(s0, s1) if i % 2 == 0 else step(s1, s0)
    ga, gb = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(ga):
        step(s0, s1)
    with torch.cuda.graph(gb):
        step(s1, s0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total = 0.0
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            e0.record(stream)
            (ga if i % 2 == 0 else gb).replay()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
    del ga, gb
    value = n * args.steps / (total * 1e-3)
    last = s1 if args.steps % 2 == 1 else s0
    finite = bool(torch.isfinite(last.particle_q).all())
    ncont = int(contacts.soft_contact_count.item())
    # end to end: host state in, one step, host state out, every step
    hx, hv = last.particle_q.cpu().pin_memory(), last.particle_qd.cpu().pin_memory()
    e2e_steps = min(args.steps, 50)
    e2e = pipelined_e2e(model, step, hx, hv, e2e_steps, device)
    cpu = None
    if not args.no_cpu_baseline:
        rate, reps, el, threads = xpbd_oracle_rate(model, w, last.particle_q.cpu().numpy(),
                                                   last.particle_qd.cpu().numpy(), budget_s=10.0)
        cpu = {"value": rate, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": f"{reps} full steps of the {n}-particle scene in {el:.1f} s (the oracle's restatement of "
                         "SolverXPBD.step: soft contacts, integrate, grid, iterations; OpenMP)"}
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "desc": w["desc"], "iterations": it, "dt": dt,
                   "grid_dims": [128, 128, 128], "graph": True, "soft_contacts": ncont,
                   "l2": "flushed (256 MiB write) before every timed step, outside the timed interval"},
        "cpu_baseline": cpu,
        "e2e": {"value": n * e2e_steps / (e2e * 1e-3), "unit": METRIC, "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 24 * n, "steps": e2e_steps,
                "how": "pinned upload of x, v, Model.collide + SolverXPBD.step, download of x, v, every step; "
                       "independent steps pipelined on upload / compute / download streams"},
        "gpu_launches": None,
        "clocks": clk.summary(),
        "finite": finite,
    }
    print(json.dumps(line), flush=True)
    return 0


def xpbd_oracle_rate(model, w, x, v, budget_s: float):
    """particle-steps/s of the oracle's XPBD step on the host cores."""
    from oracle import oracle as O

    O.build()
    md = dict(inv_mass=model.particle_inv_mass.cpu().numpy(), radius=model.particle_radius.cpu().numpy(),
              flags=model.particle_flags.cpu().numpy(), world=model.particle_world.cpu().numpy(),
              gravity=model.gravity.cpu().numpy(), v_max=model.particle_max_velocity, particle_mu=model.particle_mu,
              particle_cohesion=model.particle_cohesion, max_radius=model.particle_max_radius,
              shapes=[dict(type=sh["type"], flags=sh["flags"], world=sh["world"], pos=sh["pos"], rot=sh["rot"],
                           scale=sh["scale"], ke=sh["ke"], kd=sh["kd"], kf=sh["kf"], mu=sh["mu"])
                      for sh in model._shapes],
              soft=(model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_kf, model.soft_contact_mu,
                    model.particle_adhesion, model.soft_contact_restitution))
    it, dt = w["xpbd"]["iterations"], w["xpbd"]["dt"]
    f = np.zeros_like(x)
    t0 = time.perf_counter()
    reps = 0
    while True:
        c = O.soft_contacts_create(md["shapes"], x, md["radius"], md["flags"], world=md["world"], margin=0.01)
        xi, vi, x, v = O.xpbd_particle_step(md, x, v, f, dt, it, 0.9, contacts=c)
        reps += 1
        el = time.perf_counter() - t0
        if el > budget_s or reps >= 5:
            break
    return model.particle_count * reps / el, reps, el, O.get_threads()


def run_xpbd_reference(args):
    """The oracle's restatement of SolverXPBD.step on the same scene, all host
    threads."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    model = make_xpbd_scene(w, "cpu")
    n = model.particle_count
    rate, reps, el, threads = xpbd_oracle_rate(model, w, model.particle_q.numpy().copy(),
                                               model.particle_qd.numpy().copy(), budget_s=60.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
        "steps": reps, "warmup": 0, "ms_per_step": 1e3 * el / reps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "desc": w["desc"]},
        "cpu_baseline": {"value": rate, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{reps} full steps (oracle restatement of SolverXPBD.step, OpenMP)"},
        "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_contact_reference(args):
    """The fp32 CPU restatement of eval_particle_contact (with its grid
    build) on the same scene, all host threads."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O

    w = WORKLOADS[args.workload]
    model = make_contact_scene(w, "cpu")
    n = model.particle_count
    O.build()
    xs, vs = model.particle_q.numpy(), model.particle_qd.numpy()
    rr, fl = model.particle_radius.numpy(), model.particle_flags.numpy()
    gr = float(np.float32(2.0 * model.particle_max_radius + model.particle_cohesion))

    def step():
        O.particle_contact_forces(xs, vs, rr, fl, gr, (128, 128, 128), model.particle_ke, model.particle_kd,
                                  model.particle_kf, model.particle_mu, model.particle_cohesion,
                                  model.particle_max_radius)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    value = n * args.steps / el
    threads = O.get_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "desc": w["desc"]},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full steps (grid build + contact forces, fp32 restatement, OpenMP)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def make_raycast_sensor(model, w):
    import warnings

    from newton_sph_dev_b200.sensors import SensorRaycast

    rc = w["raycast"]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", DeprecationWarning)
        sensor = SensorRaycast(model, rc["position"], (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), rc["fov"], rc["width"],
                               rc["height"], max_distance=rc["max_distance"])
    sensor.point_camera_at(target=rc["target"], position=rc["position"], up=(0.0, 0.0, 1.0))
    return sensor


def raycast_cpu(model, sensor, x, rows: int):
    """The oracle's raycast (its own grid build included) of the sensor's
    camera at `rows` rows instead of its height: the same frustum, fewer
    rays. Returns (rays, seconds)."""
    from oracle import oracle as O

    from newton_sph_dev_b200.sensors import march_steps

    O.build()
    r = model.particle_radius.cpu().numpy()
    sr = float(model.particle_max_radius) + 1e-6
    step = 0.5 * sr
    steps = march_steps(sensor.max_distance, step)[0]
    cam = O.raycast_camera(sensor.camera_position, sensor.camera_direction, sensor.camera_up, sensor.camera_right,
                           sensor.fov_scale, sensor.aspect_ratio, sensor.width, rows, sensor.max_distance)
    t0 = time.perf_counter()
    O.raycast_particles(x, r, (128, 128, 128), cam, sr, step, steps)
    return sensor.width * rows, time.perf_counter() - t0


def run_raycast(args):
    import torch

    world, rank, local = dist_env()
    if world > 1:
        raise SystemExit("raycast_1m runs on one GPU (replicas are not wired for it)")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    w = WORKLOADS[args.workload]
    model = make_contact_scene(w, str(device))
    n = model.particle_count
    state = model.state()
    sensor = make_raycast_sensor(model, w)
    rays = sensor.width * sensor.height
    stream = torch.cuda.current_stream(device)

    def step():
        sensor.update(state, include_particles=True)

    for _ in range(max(args.warmup, 3)):
        step()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    total = build_ms = 0.0
    grid = sensor._get_particle_grid()
    sr = float(model.particle_max_radius) + 1e-6
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            ev[0].record(stream)
            grid.build(state.particle_q, sr)
            ev[1].record(stream)
            step()
            ev[2].record(stream)
            ev[2].synchronize()
            build_ms += ev[0].elapsed_time(ev[1])
            total += ev[1].elapsed_time(ev[2])
    gtotal = 0.0
    for _ in range(args.steps):
        flush.zero_()
        ev[0].record(stream)
        g.replay()
        ev[2].record(stream)
        ev[2].synchronize()
        gtotal += ev[0].elapsed_time(ev[2])
    del g
    depth = sensor.get_depth_image_numpy()
    best = min(total, gtotal)
    value = rays * args.steps / (best * 1e-3)
    # the march kernel alone: one update minus its grid build
    t_march = max(total - build_ms, 1e-9) / args.steps * 1e-3
    peak, peak_kind = load_peak()
    alg = 32 * n + 4 * rays  # gather (read x, r; write the sorted mirror) once, depth once
    roofline = {"bound": "hbm", "kernel": "k_raycast (+ gather, clamp)", "achieved": alg / t_march / 1e9,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": alg / t_march / 1e9 / peak,
                "traffic": None, "alg_bytes_per_launch": alg, "ms_per_launch": t_march * 1e3,
                "note": "the march reads the 16.8 MB cell table and the sorted mirror from L2; it is latency-bound"}
    # end to end: host positions in, depth image out, every frame; two sensors
    # so that frames pipeline on upload / compute / download streams
    sensors = {}

    def e2e_step(a, b):
        sn = sensors.setdefault(id(b), make_raycast_sensor(model, w))
        sn.update(a, include_particles=True)

    hx, hv = state.particle_q.cpu().pin_memory(), state.particle_qd.cpu().pin_memory()
    e2e_steps = min(args.steps, 50)

    def outputs(st):
        sn = sensors.setdefault(id(st), make_raycast_sensor(model, w))
        return (sn.get_depth_image(),)

    e2e = pipelined_e2e(model, e2e_step, hx, hv, e2e_steps, device, outputs=outputs)
    cpu = None
    if not args.no_cpu_baseline:
        nr, el = raycast_cpu(model, sensor, state.particle_q.cpu().numpy(), sensor.height // 8)
        from oracle import oracle as O

        cpu = {"value": nr / el, "unit": "rays/s", "cores": O.get_threads(), "kind": "port",
               "sample": f"{nr} rays (the frame's frustum at 1/8 of its rows, the grid build included) in {el:.1f} s "
                         "(fp32 restatement of the reference's march, full query at every sample, OpenMP)"}
    clocks = clk.summary()
    line = {
        "metric": "rays/s", "value": value, "unit": "rays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": best / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": n, "rays": rays, "desc": w["desc"],
                   "grid_dims": [128, 128, 128], "graph": gtotal <= total,
                   "l2": "flushed (256 MiB write) before every timed step, outside the timed interval"},
        "phase_ms_per_step": {"build": build_ms / args.steps, "march": t_march * 1e3},
        "hits": int((depth > 0).sum()), "misses": int((depth < 0).sum()),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": rays * e2e_steps / (e2e * 1e-3), "unit": "rays/s", "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 4 * rays, "steps": e2e_steps,
                "how": "pinned upload of x (and v), SensorRaycast.update, download of the depth image, every frame; "
                       "independent frames pipelined on upload / compute / download streams"},
        "gpu_launches": (grid.last_launches + 3) * args.steps,  # per timed update: build, gather, march, clamp
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_raycast_reference(args):
    """The fp32 CPU restatement of the reference's particle raycast (its own
    grid build, the full query at every march sample) on the same scene and
    camera, all host threads; each step a row subset of the frame."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    model = make_contact_scene(w, "cpu")
    sensor = make_raycast_sensor(model, w)
    x = model.particle_q.numpy()
    rays = 0
    el = 0.0
    for _ in range(args.steps):
        nr, t = raycast_cpu(model, sensor, x, sensor.height // 16)
        rays += nr
        el += t
    value = rays / el
    from oracle import oracle as O

    line = {
        "impl": "reference", "metric": "rays/s", "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": model.particle_count, "desc": w["desc"]},
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": O.get_threads(), "kind": "port",
                         "sample": f"{args.steps} x {sensor.width * (sensor.height // 16)} rays (the frame's "
                                   "frustum at 1/16 of its rows)"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=[k for k in WORKLOADS if not k.startswith("_")], default="tank_1m")
    ap.add_argument("--no-graph", action="store_true", help="time eager steps instead of graph replays")
    ap.add_argument("--weights", default=None, help="surrogate weights (.npz) for the surrogate workloads")
    ap.add_argument("--surrogate-calls", type=int, default=100,
                    help="calls of the surrogate / uncorrected / plain comparison added to the plain step's line")
    ap.add_argument("--relax", type=int, default=200,
                    help="untimed steps after the warm-up, so the timed steps run on a settled state")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shape")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    grad = "grad" in WORKLOADS[args.workload]
    if args.impl == "reference":
        if "raycast" in WORKLOADS[args.workload]:
            return run_raycast_reference(args)
        if "contact" in WORKLOADS[args.workload]:
            return run_contact_reference(args)
        if "xpbd" in WORKLOADS[args.workload]:
            return run_xpbd_reference(args)
        return run_grad_reference(args) if grad else run_reference(args)
    if "surrogate" in WORKLOADS[args.workload]:
        return run_surrogate(args)
    if "raycast" in WORKLOADS[args.workload]:
        return run_raycast(args)
    if "contact" in WORKLOADS[args.workload]:
        return run_contact(args)
    if "xpbd" in WORKLOADS[args.workload]:
        return run_xpbd(args)
    return run_grad(args) if grad else run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
