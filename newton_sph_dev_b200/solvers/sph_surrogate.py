"""Learned surrogate step for SolverSPH: a larger time step whose
acceleration is corrected per particle by a small MLP.

The reference has no learned components; this is the "surrogate" form that
builds on the plain step. Pieces:

- :class:`SurrogateModel`: the MLP (16 -> 64 -> 64 -> 3, SiLU) as one fp32
  device buffer in the library's layout (``nsph_mlp_model_floats``); the
  kernels round weights and activations to bf16 and accumulate in fp32 on
  the tcgen05 tensor cores.
- :func:`generate_training_data`: runs the plain solver and records, at every
  ``substeps``-th step, the 16 neighbour features of each particle and the
  acceleration correction that makes one step of ``substeps * dt`` land
  where ``substeps`` plain steps landed.
- :class:`SurrogateTrainer`: Adam on the library's gradient kernel
  (``nsph_mlp_gradient`` / ``nsph_mlp_adam``).
- :class:`SurrogateSPH`: the stepper. Each call advances ``substeps * dt``:
  one surrogate step, or ``substeps`` plain steps when the surrogate is
  suspended. The plain step is the fallback and the yardstick: the mean
  compression error e = mean_i max(0, rho_i/rho0 - 1) of every surrogate step
  is accumulated on the device; every ``window`` calls the host reads the
  window's worst value (one copy). Above ``threshold`` (or NaN) the window is
  rejected: with ``rollback`` (the default) the state saved at the window's
  start is restored and the window is run again with plain steps, so every
  committed surrogate window stays within the threshold; the surrogate is
  then suspended for the next window(s), longer after consecutive failures.

Every quantity the network sees or predicts is dimensionless (lengths / h,
velocities / c0, accelerations h / c0^2 with c0^2 = B gamma / rho0), so a
model trained at one resolution applies at another with the same
dimensionless step dt c0 / h.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import torch

from .. import _lib
from .sph import SPHConfig, SolverSPH

FEATURES = (
    "rho/rho0", "rho/rho0-1", "mx", "my", "mz", "dvx", "dvy", "dvz", "ax", "ay", "az", "m2", "shepard", "div_v",
    "p", "|a|",
)
N_IN, N_HID, N_OUT = 16, 64, 3
W1, B1, W2, B2, W3, B3 = 0, 1024, 1088, 5184, 5248, 5440
N_PARAMS = 5443
IN_MEAN, IN_INV_STD, OUT_MEAN, OUT_STD = 5448, 5464, 5480, 5484
MODEL_FLOATS = 5488
# weights trained by newton_sph_dev_b200.train_surrogate (defaults: 200
# trajectories of 32,768 particles at spacing 0.01 m, dt 1e-4 s, 4 substeps)
PRETRAINED = Path(__file__).resolve().parents[1] / "surrogate_weights.npz"


def c0_squared(config: SPHConfig) -> float:
    """c0^2 as the kernels derive it from the fp32 parameters (B gamma / rho0)."""
    c = config.constants(0.0, 1.0)["f32"]
    return float(np.float32(c["eos_b"]) * np.float32(c["eos_gamma"]) * np.float32(c["inv_rho0"]))


def accel_scale(config: SPHConfig) -> float:
    """c0^2 / h: the unit of the network's dimensionless acceleration."""
    return c0_squared(config) / float(np.float32(config.smoothing_length))


class SurrogateModel:
    """The MLP's parameters in one fp32 device buffer (library layout)."""

    def __init__(self, device: str | torch.device = "cuda:0", seed: int = 0):
        self.device = torch.device(device)
        L = _lib.load()
        if L.nsph_mlp_model_floats() != MODEL_FLOATS:
            raise RuntimeError("libnsph.so model layout does not match this module")
        self.buf = torch.zeros(MODEL_FLOATS, dtype=torch.float32, device=self.device)
        g = torch.Generator().manual_seed(seed)
        for off, fan_in, fan_out in ((W1, N_IN, N_HID), (W2, N_HID, N_HID), (W3, N_HID, N_OUT)):
            bound = math.sqrt(6.0 / (fan_in + fan_out))
            w = (torch.rand(fan_in * fan_out, generator=g) * 2 - 1) * bound
            self.buf[off:off + fan_in * fan_out] = w.to(self.device)
        self.buf[IN_INV_STD:IN_INV_STD + N_IN] = 1.0
        self.buf[OUT_STD:OUT_STD + N_OUT] = 1.0
        self.meta: dict = {}

    # ---- views -------------------------------------------------------
    @property
    def w1(self):
        return self.buf[W1:B1].view(N_IN, N_HID)

    @property
    def b1(self):
        return self.buf[B1:W2]

    @property
    def w2(self):
        return self.buf[W2:B2].view(N_HID, N_HID)

    @property
    def b2(self):
        return self.buf[B2:W3]

    @property
    def w3(self):
        return self.buf[W3:B3].view(N_HID, N_OUT)

    @property
    def b3(self):
        return self.buf[B3:N_PARAMS]

    def set_normalization(self, in_mean, in_std, out_mean, out_std) -> None:
        t = lambda a: torch.as_tensor(a, dtype=torch.float32, device=self.device)
        self.buf[IN_MEAN:IN_MEAN + N_IN] = t(in_mean)
        self.buf[IN_INV_STD:IN_INV_STD + N_IN] = 1.0 / torch.clamp(t(in_std), min=1e-12)
        self.buf[OUT_MEAN:OUT_MEAN + N_OUT] = t(out_mean)
        self.buf[OUT_STD:OUT_STD + N_OUT] = t(out_std)

    def zero_correction(self) -> None:
        """Make the network's output exactly zero (W3 = b3 = out_mean = 0):
        the surrogate step is then the plain step at the large dt."""
        self.buf[W3:N_PARAMS] = 0.0
        self.buf[OUT_MEAN:OUT_MEAN + N_OUT] = 0.0

    # ---- evaluation ---------------------------------------------------
    def forward(self, features: torch.Tensor) -> torch.Tensor:
        """De-normalised outputs (n, 3) of raw features (n, 16) on the tensor cores."""
        f = features.to(device=self.device, dtype=torch.float32).contiguous()
        n = int(f.shape[0])
        out = torch.empty((n, N_OUT), dtype=torch.float32, device=self.device)
        err = torch.zeros(1, dtype=torch.int32, device=self.device)
        L = _lib.load()
        _lib.check(L.nsph_mlp_forward(self.device.index or 0, self.buf.data_ptr(), f.data_ptr(), n, out.data_ptr(),
                                      err.data_ptr(), _lib.stream_handle(self.device)), "SurrogateModel.forward")
        return out

    def reference_forward(self, features: torch.Tensor) -> torch.Tensor:
        """The same network in torch fp32 with the kernels' bf16 roundings
        (inputs, weights, hidden activations); for checks."""
        bf = lambda t: t.to(torch.bfloat16).to(torch.float32)
        f = features.to(self.device, torch.float32)
        x = bf((f - self.buf[IN_MEAN:IN_MEAN + N_IN]) * self.buf[IN_INV_STD:IN_INV_STD + N_IN])
        h1 = bf(torch.nn.functional.silu(x @ bf(self.w1) + self.b1))
        h2 = bf(torch.nn.functional.silu(h1 @ bf(self.w2) + self.b2))
        y = h2 @ bf(self.w3) + self.b3
        return y * self.buf[OUT_STD:OUT_STD + N_OUT] + self.buf[OUT_MEAN:OUT_MEAN + N_OUT]

    # ---- persistence --------------------------------------------------
    def save(self, path) -> None:
        meta = {k: (v if isinstance(v, (int, float, str)) else str(v)) for k, v in self.meta.items()}
        np.savez(path, buf=self.buf.detach().cpu().numpy(), meta=np.array([repr(meta)]))

    @classmethod
    def pretrained(cls, device: str | torch.device = "cuda:0") -> "SurrogateModel":
        """The weights shipped with the package (PRETRAINED)."""
        return cls.load(PRETRAINED, device)

    @classmethod
    def load(cls, path, device: str | torch.device = "cuda:0") -> "SurrogateModel":
        d = np.load(path, allow_pickle=False)
        m = cls(device)
        buf = d["buf"]
        if buf.shape != (MODEL_FLOATS,):
            raise ValueError(f"{path}: model buffer has shape {buf.shape}, expected ({MODEL_FLOATS},)")
        m.buf.copy_(torch.from_numpy(buf.astype(np.float32)))
        m.meta = {"file": str(path), "saved_meta": str(d["meta"][0]) if "meta" in d else ""}
        return m


class SurrogateTrainer:
    """Adam on the library's hand-written gradient kernel (mean squared
    error on normalised targets)."""

    def __init__(self, model: SurrogateModel, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8):
        self.model = model
        self.lr, self.betas, self.eps = lr, betas, eps
        dev = model.device
        self.m = torch.zeros(N_PARAMS, dtype=torch.float32, device=dev)
        self.v = torch.zeros(N_PARAMS, dtype=torch.float32, device=dev)
        self.grad = torch.zeros(N_PARAMS + 1, dtype=torch.float32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.t = 0
        self._partials = None

    def gradient(self, features: torch.Tensor, targets: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
        """grad (5443 + 1: the gradient in model order, then the loss) over the rows idx."""
        L = _lib.load()
        dev = self.model.device
        batch = int(idx.numel())
        ctas = L.nsph_mlp_gradient_ctas(dev.index or 0, batch)
        if self._partials is None or self._partials.shape[0] < ctas:
            self._partials = torch.empty((ctas, N_PARAMS + 1), dtype=torch.float32, device=dev)
        idx = idx.to(device=dev, dtype=torch.int32).contiguous()
        features = features.contiguous()
        targets = targets.contiguous()
        _lib.check(L.nsph_mlp_gradient(dev.index or 0, self.model.buf.data_ptr(), features.data_ptr(),
                                       targets.data_ptr(), idx.data_ptr(), batch, self._partials.data_ptr(),
                                       int(self._partials.shape[0]), self.grad.data_ptr(), self.err.data_ptr(),
                                       _lib.stream_handle(dev)), "SurrogateTrainer.gradient")
        return self.grad

    def step(self, features: torch.Tensor, targets: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
        """One Adam step on the batch rows idx; returns the batch loss (device scalar)."""
        self.gradient(features, targets, idx)
        self.t += 1
        L = _lib.load()
        dev = self.model.device
        _lib.check(L.nsph_mlp_adam(dev.index or 0, self.model.buf.data_ptr(), self.grad.data_ptr(),
                                   self.m.data_ptr(), self.v.data_ptr(), float(self.lr), float(self.betas[0]),
                                   float(self.betas[1]), float(self.eps), self.t, _lib.stream_handle(dev)),
                   "SurrogateTrainer.step")
        return self.grad[N_PARAMS]


# ---------------------------------------------------------------------------
# training data from plain trajectories
# ---------------------------------------------------------------------------
def _lattice_model(shape, spacing, jitter_seed, vel_std, vel_seed, device):
    from ..sim import ModelBuilder

    rng = np.random.default_rng(jitter_seed)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in shape], indexing="ij"), -1).reshape(-1, 3)
    x = ((g + 0.5) * spacing + rng.uniform(-0.1 * spacing, 0.1 * spacing, g.shape)).astype(np.float32)
    v = np.random.default_rng(vel_seed).normal(0.0, vel_std, x.shape).astype(np.float32) if vel_std > 0 else \
        np.zeros_like(x)
    b = ModelBuilder()
    b.add_particles(pos=x.tolist(), vel=v.tolist(), mass=[1000.0 * spacing**3] * len(x))
    return b.finalize(device)


def surrogate_targets(config: SPHConfig, dt_big: float, x0, v0, x1, acc, gravity, box_margin: float = 1e-6):
    """Dimensionless correction (n, 3) that moves one step of dt_big from
    (x0, v0) to x1, and the mask of usable rows.

    The surrogate step is v' = v0 + (a + da + g) dt + eps dv, x' = x0 + v' dt,
    so da = ((x1 - x0) / dt - v0 - eps dv) / dt - a - g."""
    a, dv = acc[:, 0:3], acc[:, 3:6]
    vbar = (x1 - x0) / dt_big
    da = (vbar - v0 - config.xsph * dv) / dt_big - a - gravity
    target = da / accel_scale(config)
    ok = torch.isfinite(target).all(dim=1)
    if config.box_lo is not None and config.box_hi is not None:
        lo = torch.tensor(config.box_lo, dtype=x1.dtype, device=x1.device) + box_margin
        hi = torch.tensor(config.box_hi, dtype=x1.dtype, device=x1.device) - box_margin
        ok &= ((x1 > lo) & (x1 < hi)).all(dim=1)
    return target, ok


def generate_training_data(trajectories: int = 200, shape=(32, 32, 32), spacing: float = 0.01, dt: float = 1e-4,
                           substeps: int = 4, samples_per_trajectory: int = 10, keep_fraction: float = 0.125,
                           vel_scale=(0.0, 0.5), box=(1.0, 1.0, 1.0), seed: int = 0, stride: int = 1,
                           device: str | torch.device = "cuda:0"):
    """Features (N, 16) and dimensionless targets (N, 3) from plain
    trajectories of jittered lattice blocks (32^3 = 32,768 particles by
    default, in a 1 m box, velocities N(0, s^2) per component with s uniform
    in vel_scale). Each trajectory runs samples_per_trajectory x stride x
    substeps plain steps of dt; every (stride x substeps)-th state is a
    sample (whose target spans the next substeps steps), of which a random
    keep_fraction of the particles is kept. A stride above 1 spreads the
    samples over a longer span of the flow (the block's collapse and
    splash) at the same number of rows.

    Returns (features, targets, info)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=torch.device(device)).manual_seed(seed)
    feats, targs = [], []
    cfg = SPHConfig(smoothing_length=2 * spacing, box_lo=(0.0, 0.0, 0.0), box_hi=box)
    dt_big = substeps * dt
    kept = 0
    for _ in range(trajectories):
        vs = float(rng.uniform(*vel_scale))
        model = _lattice_model(shape, spacing, int(rng.integers(1 << 30)), vs, int(rng.integers(1 << 30)), device)
        solver = SolverSPH(model, cfg)
        solver.enable_surrogate()
        n = model.particle_count
        grav = model.gravity[0].to(torch.float32)
        x = model.particle_q.clone()
        v = model.particle_qd.clone()
        p_small = solver.step_params(dt)
        p_big = solver.step_params(dt_big)
        feat = torch.empty((n, N_IN), dtype=torch.float32, device=model.device)
        acc = torch.empty((n, 6), dtype=torch.float32, device=model.device)
        tx = torch.empty((substeps, n, 3), dtype=torch.float32, device=model.device)
        tv = torch.empty_like(tx)
        for _ in range(samples_per_trajectory):
            solver.features_raw(x, v, feat, acc, params=p_big)
            solver.rollout_raw(x, v, tx, tv, p_small)
            x1 = tx[-1]
            target, ok = surrogate_targets(cfg, dt_big, x, v, x1, acc, grav)
            sel = ok & (torch.rand(n, device=model.device, generator=gen) < keep_fraction)
            feats.append(feat[sel].clone())
            targs.append(target[sel].clone())
            kept += int(sel.sum())
            x, v = x1.clone(), tv[-1].clone()
            for _ in range(stride - 1):  # unrecorded plain steps to the next sample
                solver.rollout_raw(x, v, tx, tv, p_small)
                x, v = tx[-1].clone(), tv[-1].clone()
    features = torch.cat(feats)
    targets = torch.cat(targs)
    info = {"trajectories": trajectories, "particles": int(np.prod(shape)), "spacing": spacing, "dt": dt,
            "substeps": substeps, "samples_per_trajectory": samples_per_trajectory,
            "plain_steps_per_trajectory": samples_per_trajectory * stride * substeps, "stride": stride,
            "keep_fraction": keep_fraction, "vel_scale": tuple(vel_scale), "rows": kept, "seed": seed}
    return features, targets, info


def fit_normalization(model: SurrogateModel, features: torch.Tensor, targets: torch.Tensor) -> None:
    fm, fs = features.mean(0), features.std(0)
    fs = torch.where(fs > 1e-8, fs, torch.ones_like(fs))
    tm, ts = targets.mean(0), targets.std(0)
    ts = torch.where(ts > 1e-12, ts, torch.ones_like(ts))
    model.set_normalization(fm, fs, tm, ts)


def train(model: SurrogateModel, features: torch.Tensor, targets: torch.Tensor, iters: int = 2000,
          batch: int = 65536, lr: float = 1e-3, seed: int = 0, val_fraction: float = 0.05, log_every: int = 0):
    """Fit the model (normalisation from the data, then Adam with a cosine
    learning-rate decay). Returns a dict with the training and validation
    losses (normalised MSE; 1.0 = predicting the mean)."""
    g = torch.Generator(device=features.device).manual_seed(seed)
    n = int(features.shape[0])
    perm = torch.randperm(n, generator=g, device=features.device)
    nval = max(1, int(n * val_fraction))
    val_idx, train_idx = perm[:nval], perm[nval:]
    fit_normalization(model, features[train_idx], targets[train_idx])
    opt = SurrogateTrainer(model, lr=lr)
    features = features.contiguous()
    targets = targets.contiguous()
    hist = []
    for it in range(iters):
        opt.lr = lr * 0.5 * (1 + math.cos(math.pi * it / max(1, iters)))
        bi = train_idx[torch.randint(0, train_idx.numel(), (batch,), generator=g, device=features.device)]
        loss = opt.step(features, targets, bi)
        if log_every and (it % log_every == 0 or it == iters - 1):
            hist.append((it, float(loss.item())))
    val_loss = float(opt.gradient(features, targets, val_idx)[N_PARAMS].item())
    train_loss = float(opt.gradient(features, targets, train_idx[:min(train_idx.numel(), 1 << 20)])[N_PARAMS].item())
    return {"train_loss": train_loss, "val_loss": val_loss, "history": hist, "rows": n, "iters": iters,
            "batch": batch, "lr": lr}


# ---------------------------------------------------------------------------
# the stepper: surrogate steps with the plain step as fallback
# ---------------------------------------------------------------------------
class FallbackMonitor:
    """Host side of the fallback rule (no device access): given the worst
    compression error of each window of surrogate steps, decide whether the
    next window runs the surrogate or the plain step. A window above the
    threshold suspends the surrogate for `cooldown` windows; with `backoff`,
    each further failure in a row doubles that (up to `max_cooldown`), and a
    window that passes resets it."""

    def __init__(self, threshold: float = 0.01, cooldown: int = 1, backoff: bool = False, max_cooldown: int = 64):
        self.threshold = threshold
        self.cooldown = cooldown
        self.backoff = bool(backoff)
        self.max_cooldown = int(max_cooldown)
        self.suspended = 0
        self.trips = 0
        self.in_a_row = 0

    def use_surrogate(self) -> bool:
        return self.suspended == 0

    def end_window(self, worst: float | None) -> bool:
        """worst: the window's max compression error (None for a plain
        window). Returns True when a surrogate window failed (trip)."""
        if worst is None:
            self.suspended = max(0, self.suspended - 1)
            return False
        if not (worst <= self.threshold):  # NaN counts as a trip
            self.trips += 1
            self.in_a_row += 1
            c = self.cooldown * (2 ** (self.in_a_row - 1) if self.backoff else 1)
            self.suspended = min(c, max(self.max_cooldown, self.cooldown))
            return True
        self.in_a_row = 0
        return False


class SurrogateSPH:
    """Advance a SolverSPH model by substeps x dt per call: one surrogate step
    of dt_big = substeps x dt, or substeps plain steps while the surrogate is
    suspended by the fallback rule (see the module docstring). A window in
    which a tensor-core wait gave up (NSPH_STATUS_SURROGATE_TIMEOUT) counts as
    failed, like one above the threshold.

    With ``rollback`` (default) a failed window is replaced: the call that
    ends it restores the state saved when the window began (two device
    copies per window) and runs the window's calls again as plain steps, so
    the state it returns is the plain trajectory's; states returned by the
    window's earlier calls were speculative. Without it, a failed window is
    kept and only the next window(s) run plain steps. ``backoff`` doubles the
    suspension after each further failure in a row (see FallbackMonitor)."""

    def __init__(self, solver: SolverSPH, model: SurrogateModel, substeps: int = 4, threshold: float = 0.01,
                 window: int = 10, cooldown: int = 1, graphs: bool = False, rollback: bool = True,
                 backoff: bool = True):
        if solver.batched:
            raise ValueError("the surrogate needs a single-world solver")
        self.solver = solver
        self.model = model
        self.substeps = int(substeps)
        self.window = int(window)
        self.monitor = FallbackMonitor(threshold, cooldown, backoff=backoff)
        self.rollback = bool(rollback)
        self._ckpt = None
        self.rollbacks = 0
        self.committed_compression = 0.0  # sum of e over the surrogate steps kept
        self.rejected_worst: list[float] = []
        self._stats_at_window = 0.0
        solver.enable_surrogate()
        self.stats = torch.zeros(4, dtype=torch.float32, device=solver.model.device)
        self._traj = None
        self.calls = 0
        self.surrogate_steps = 0
        self.fallback_calls = 0
        self.timeouts = 0
        self.window_worst: list[float] = []
        self._window_mode = True
        self.acc_scale = accel_scale(solver.config)
        self.graphs = bool(graphs)  # replay each (state_in, state_out, dt) surrogate step from a CUDA graph
        self._graphs: dict = {}
        self.launches_per_step = 0

    def step(self, state_in, state_out, dt: float) -> None:
        """Advance state_in by substeps x dt into state_out."""
        if self.calls % self.window == 0:
            self._window_mode = self.monitor.use_surrogate()
            if self._window_mode and self.rollback:  # the state the window may return to
                if self._ckpt is None:
                    self._ckpt = (torch.empty_like(state_in.particle_q), torch.empty_like(state_in.particle_qd))
                self._ckpt[0].copy_(state_in.particle_q)
                self._ckpt[1].copy_(state_in.particle_qd)
        if self._window_mode:
            self._surrogate_step(state_in, state_out, dt)
            self.surrogate_steps += 1
        else:
            self._plain_call(state_in.particle_q, state_in.particle_qd, state_out, dt)
            self.fallback_calls += 1
        self.calls += 1
        if self.calls % self.window == 0:
            self._end_window(state_out, dt)

    def reset_counters(self) -> None:
        """Start the counters, the statistics and the fallback rule afresh
        (captured graphs are kept)."""
        self.stats.zero_()
        self.calls = self.surrogate_steps = self.fallback_calls = self.timeouts = self.rollbacks = 0
        self.window_worst = []
        self.rejected_worst = []
        self.committed_compression = 0.0
        self._stats_at_window = 0.0
        self.monitor.suspended = self.monitor.trips = self.monitor.in_a_row = 0

    def _plain_steps(self, q, qd, state_out, dt):
        """substeps plain steps of dt from (q, qd) into state_out, through two
        scratch states (each step's velocity output starts as its input, so
        inactive particles keep their velocity, as in nsph_sph_rollout)."""
        if self._traj is None:
            self._traj = tuple(torch.empty_like(q) for _ in range(4))
        p = self.solver.step_params(dt)
        cur_q, cur_qd = q, qd
        for i in range(self.substeps):
            last = i == self.substeps - 1
            oq, oqd = (state_out.particle_q, state_out.particle_qd) if last else self._traj[2 * (i % 2):2 * (i % 2) + 2]
            oqd.copy_(cur_qd)
            self.solver.step_raw(cur_q, cur_qd, oq, oqd, p)
            cur_q, cur_qd = oq, oqd

    def _plain_call(self, q, qd, state_out, dt):
        """substeps plain steps of dt from (q, qd) into state_out (replayed
        from a CUDA graph per (buffers, dt) with ``graphs``)."""
        if not self.graphs:
            self._plain_steps(q, qd, state_out, dt)
            return
        key = ("plain", q.data_ptr(), qd.data_ptr(), state_out.particle_q.data_ptr(),
               state_out.particle_qd.data_ptr(), float(dt))
        g = self._graphs.get(key)
        if g is None:  # run eagerly this time, then capture for the next calls
            self._plain_steps(q, qd, state_out, dt)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._plain_steps(q, qd, state_out, dt)
            self._graphs[key] = g
            # the capture ran nothing: state_out holds the eager result
            return
        g.replay()

    def _surrogate_call(self, state_in, state_out, dt):
        self.solver.step_surrogate_raw(state_in.particle_q, state_in.particle_qd, state_out.particle_q,
                                       state_out.particle_qd, self.solver.step_params(self.substeps * dt),
                                       self.model, self.acc_scale, self.stats)

    def _surrogate_step(self, state_in, state_out, dt):
        if not self.graphs:
            self._surrogate_call(state_in, state_out, dt)
            self.launches_per_step = self.solver.last_launches
            return
        key = (state_in.particle_q.data_ptr(), state_in.particle_qd.data_ptr(), state_out.particle_q.data_ptr(),
               state_out.particle_qd.data_ptr(), float(dt))
        g = self._graphs.get(key)
        if g is None:  # run eagerly this time, then capture for the next calls
            self._surrogate_call(state_in, state_out, dt)
            self.launches_per_step = self.solver.last_launches
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._surrogate_call(state_in, state_out, dt)
            self._graphs[key] = g
            return
        g.replay()

    def _end_window(self, state_out, dt: float) -> None:
        if not self._window_mode:
            self.monitor.end_window(None)
            return
        s = self.stats.cpu()  # one copy: worst, steps, running sum
        worst = float(s[1])
        window_sum = float(s[3]) - self._stats_at_window
        self._stats_at_window = float(s[3])
        # a tensor-core wait that gave up integrated part of a step
        # without the correction: count the window as failed
        if self.solver.status() & _lib.NSPH_STATUS_SURROGATE_TIMEOUT:
            self.timeouts += 1
            self.solver.reset_status()
            worst = float("nan")
        self.window_worst.append(worst)
        failed = self.monitor.end_window(worst)
        self.stats[1:3].zero_()
        if failed and self.rollback:
            # replace the window: plain steps from the state it began with
            self.rollbacks += 1
            self.rejected_worst.append(worst)
            self.surrogate_steps -= self.window
            self.fallback_calls += self.window
            q, qd = self._ckpt
            for i in range(self.window):
                self._plain_call(q, qd, state_out, dt)
                if i + 1 < self.window:  # the next call starts from this one's result
                    q.copy_(state_out.particle_q)
                    qd.copy_(state_out.particle_qd)
        else:
            self.committed_compression += window_sum

    def committed_window_worst(self) -> float:
        """Worst step compression over the kept surrogate windows."""
        kept = [w for w in self.window_worst if w == w and w <= self.monitor.threshold] if self.rollback \
            else self.window_worst
        return float(max(kept or [0.0]))

    def mean_compression(self) -> float:
        """Mean compression error over the surrogate steps kept so far, as of
        the last completed window."""
        return self.committed_compression / max(1, self.surrogate_steps - (self.calls % self.window
                                                                              if self._window_mode else 0))


__all__ = ["FEATURES", "FallbackMonitor", "SurrogateModel", "SurrogateSPH", "SurrogateTrainer", "accel_scale",
           "generate_training_data", "surrogate_targets", "train"]
