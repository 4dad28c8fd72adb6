"""Train the surrogate step's MLP on plain-solver trajectories and evaluate
it on a held-out scene.

    python -m newton_sph_dev_b200.train_surrogate --out weights.npz [--report report.json]

Data: `--trajectories` (200) jittered 32^3 lattice blocks (32,768 particles,
spacing 0.01 m, h = 0.02 m, 1 m box, rho0 = 1000, Tait gamma = 7, c0 = 20
m/s, XSPH 0.01), velocity scale uniform in [0, 0.5] m/s, plain steps of
dt = 1e-4 s; every 4th state is a sample whose target is the acceleration
correction that lets one step of 4 dt land where 4 plain steps landed.
Training: Adam on the library's tcgen05 gradient kernel, cosine learning-rate
decay. Evaluation (held-out seed): a rollout of surrogate steps, and of
uncorrected steps of 4 dt, against the plain rollout of the same simulated
time; position error in units of h and the mean compression error
mean_i max(0, rho_i/rho0 - 1).
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .solvers import SolverSPH
from .solvers.sph_surrogate import (SurrogateModel, SurrogateSPH, _lattice_model, generate_training_data, train)


def save_training_data(path, features: torch.Tensor, targets: torch.Tensor, info: dict) -> None:
    """Features (N, 16), targets (N, 3) and the generator's settings as one .npz."""
    np.savez(path, features=features.detach().cpu().numpy(), targets=targets.detach().cpu().numpy(),
             info=np.array(json.dumps(info)))


def load_training_data(path, device="cuda:0"):
    """(features, targets, info) of a file written by save_training_data."""
    with np.load(path, allow_pickle=False) as d:
        feats = torch.from_numpy(d["features"]).to(device)
        targs = torch.from_numpy(d["targets"]).to(device)
        info = json.loads(str(d["info"]))
    if feats.ndim != 2 or targs.ndim != 2 or feats.shape[0] != targs.shape[0]:
        raise ValueError(f"{path}: features {tuple(feats.shape)} and targets {tuple(targs.shape)} do not pair up")
    return feats, targs, info


def evaluate(model: SurrogateModel, shape=(32, 32, 32), spacing=0.01, dt=1e-4, substeps=4, macro_steps=50,
             vel_std=0.25, seed=12345, device="cuda:0") -> dict:
    """Surrogate and uncorrected large steps against plain steps on one held-out scene."""
    from .solvers.sph import SPHConfig

    cfg = SPHConfig(smoothing_length=2 * spacing, box_lo=(0.0, 0.0, 0.0), box_hi=(1.0, 1.0, 1.0))
    rng = np.random.default_rng(seed)
    scene = _lattice_model(shape, spacing, int(rng.integers(1 << 30)), vel_std, int(rng.integers(1 << 30)), device)
    n = scene.particle_count
    out = {"particles": n, "macro_steps": macro_steps, "substeps": substeps, "dt": dt, "vel_std": vel_std}
    results = {}
    diverged: dict = {}
    zero = SurrogateModel(device)
    zero.zero_correction()
    for name, m in (("plain", None), ("surrogate", model), ("uncorrected", zero)):
        solver = SolverSPH(scene, cfg)
        s0, s1 = scene.state(), scene.state()
        rho = torch.empty(n, device=scene.device)
        comp = []
        if m is None:
            for _ in range(macro_steps * substeps):
                solver.step(s0, s1, None, None, dt)
                s0, s1 = s1, s0
        else:
            st = SurrogateSPH(solver, m, substeps=substeps, threshold=float("inf"), window=1)
            for k in range(macro_steps):
                st.step(s0, s1, dt)
                s0, s1 = s1, s0
                worst = st.window_worst[-1]
                if not (worst < 1.0) and name not in diverged:  # compression above 100%, or not finite
                    diverged[name] = k
            comp.append(st.mean_compression())
        solver.features_raw(s0.particle_q, s0.particle_qd, rho_out=rho, params=solver.step_params(dt))
        final_comp = float(torch.clamp(rho / 1000.0 - 1.0, min=0).mean())
        results[name] = (s0.particle_q.clone(), final_comp, comp[0] if comp else None)
    ref = results["plain"][0]
    h = 2 * spacing
    for name, (x, fc, mc) in results.items():
        d = (x - ref).norm(dim=1) / h
        out[name] = {"rms_error_h": float(d.pow(2).mean().sqrt()), "max_error_h": float(d.max()),
                     "final_compression": fc, "mean_step_compression": mc,
                     "finite": bool(torch.isfinite(x).all()), "diverged_at_step": diverged.get(name)}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", default=None)
    ap.add_argument("--trajectories", type=int, default=200)
    ap.add_argument("--samples", type=int, default=10, help="samples (of `substeps` plain steps) per trajectory")
    ap.add_argument("--keep", type=float, default=0.125, help="fraction of particles kept per sample")
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--substeps", type=int, default=4,
                    help="plain steps of 1e-4 s per surrogate step (4: dt c0/h = 0.4; 8: 0.8)")
    ap.add_argument("--stride", type=int, default=1,
                    help="surrogate steps between samples (1: consecutive; larger spreads a trajectory's samples "
                         "over more of the flow)")
    ap.add_argument("--eval-steps", type=int, default=50, help="surrogate steps of the held-out rollout")
    ap.add_argument("--device", default="cuda:0")
    ap.add_argument("--save-data", default=None, help="write the generated features and targets to this .npz")
    ap.add_argument("--load-data", default=None, help="train on the features and targets of this .npz instead of "
                                                       "generating them")
    args = ap.parse_args(argv)
    t0 = time.time()
    if args.load_data:
        feats, targs, info = load_training_data(args.load_data, args.device)
    else:
        feats, targs, info = generate_training_data(trajectories=args.trajectories,
                                                    samples_per_trajectory=args.samples, keep_fraction=args.keep,
                                                    seed=args.seed, device=args.device, substeps=args.substeps,
                                                    stride=args.stride)
    if args.save_data:
        save_training_data(args.save_data, feats, targs, info)
    t_data = time.time() - t0
    model = SurrogateModel(args.device, seed=args.seed)
    t0 = time.time()
    res = train(model, feats, targs, iters=args.iters, batch=args.batch, lr=args.lr, seed=args.seed,
                log_every=max(1, args.iters // 10))
    torch.cuda.synchronize()
    t_train = time.time() - t0
    model.meta = {"data": json.dumps(info), "train_loss": res["train_loss"], "val_loss": res["val_loss"],
                  "iters": args.iters, "batch": args.batch, "lr": args.lr}
    model.save(args.out)
    report = {"data": info, "data_seconds": t_data, "train_seconds": t_train, "train": res,
              "eval": evaluate(model, device=args.device, substeps=args.substeps, macro_steps=args.eval_steps)}
    text = json.dumps(report, indent=1)
    print(text)
    if args.report:
        with open(args.report, "w") as f:
            f.write(text)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
