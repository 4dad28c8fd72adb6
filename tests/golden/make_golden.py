"""Generate tests/golden/sph_small.npz: a small seeded WCSPH case with the
oracle's answers (grid arrays, neighbour lists, one fp32 step, one fp64
step). The reference has no SPH and its HashGrid lives in the absent
warp-lang, so these fixtures come from the CPU oracle; they pin the oracle
and the device against regressions across machines.

Run:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE.parent))


def make_case():
    from conftest import lattice_scene

    model, cfg = lattice_scene((6, 5, 4), spacing=0.01, vel_std=0.2, seed=7, register=False)
    n = model.particle_count
    rng = np.random.default_rng(9)
    flags = np.ones(n, np.int32)
    flags[rng.choice(n, 5, replace=False)] = 0
    mass = model.particle_mass.numpy().copy()
    mass[rng.choice(n, 4, replace=False)] = 0.0
    inv = np.divide(1.0, mass, out=np.zeros_like(mass), where=mass != 0).astype(np.float32)
    f_ext = rng.normal(0, 1e-4, (n, 3)).astype(np.float32)
    return dict(x=model.particle_q.numpy().copy(), v=model.particle_qd.numpy().copy(), mass=mass, inv_mass=inv,
                flags=flags, world=model.particle_world.numpy().copy(), gravity=model.gravity.numpy().copy(),
                f_ext=f_ext), cfg


def answers(case, cfg, dt=1e-4, v_max=1e5):
    from oracle import oracle as O

    consts = cfg.constants(dt, v_max)
    dims = cfg.resolved_grid_dims()
    g = O.grid_build(case["x"], float(consts["f32"]["cell_width"]), dims)
    off, ids = O.sph_neighbors(consts["f32"], dims, case["x"], case["flags"])
    out = {f"grid_{k}": v for k, v in g.items()}
    out["nbr_offsets"] = off
    out["nbr_ids"] = ids
    v_init = np.full_like(case["v"], -3.0)
    for prec in ("f32", "f64"):
        r = O.sph_step(consts, dims, case["x"], case["v"], case["mass"], case["inv_mass"], case["flags"],
                       case["world"], case["gravity"], f_ext=case["f_ext"], v_out_init=v_init, precision=prec)
        for k in ("x", "v", "rho", "p", "a"):
            out[f"{prec}_{k}"] = r[k]
    out["grid_dims"] = np.array(dims, np.int32)
    out["dt"] = np.float64(dt)
    return out


def main():
    from oracle import oracle as O

    O.build()
    case, cfg = make_case()
    ans = answers(case, cfg)
    np.savez_compressed(HERE / "sph_small.npz", **{f"in_{k}": v for k, v in case.items()}, **ans)
    print(f"wrote {HERE / 'sph_small.npz'}: {len(case['x'])} particles, {len(ans['nbr_ids'])} neighbour entries")


if __name__ == "__main__":
    main()
