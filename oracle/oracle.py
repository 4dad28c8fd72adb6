"""CPU oracle for the particle-fluid hot path — ctypes wrapper of liboracle.so
plus pure-Python restatements for small cases.

TEST INFRASTRUCTURE ONLY. This module is the checker: only the tests, the
smoke check (``__graft_entry__.smoke``) and the benchmark's CPU-baseline leg
may import it, and never as the thing measured or shipped.

What it restates (reference paths inside the Newton source tree):
  - Warp HashGrid build/query (external warp-lang 1.14.0.dev20260511; call
    sites newton/_src/sim/builder.py:9853,
    newton/_src/solvers/xpbd/solver_xpbd.py:139,315-319,
    newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71);
  - integrate_particles, newton/_src/solvers/solver.py:10-47;
  - the lattice generator ModelBuilder.add_particle_grid,
    newton/_src/sim/builder.py:8085-8096 (``lattice_py``);
  - the WCSPH step (published methods; the reference has no SPH).

Parity status: UNPINNED against the reference itself — the reference ships
no golden vectors for HashGrid or particle dynamics, cannot run here (no
warp-lang) and has no SPH. The oracle is pinned by analytic known answers and
brute-force restatements instead (tests/test_oracle.py).
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class SphParams32(ctypes.Structure):
    """Layout of nsph_sph_params (include/nsph.h)."""

    _fields_ = [
        ("h", ctypes.c_float),
        ("h2", ctypes.c_float),
        ("inv_h", ctypes.c_float),
        ("cell_width", ctypes.c_float),
        ("cell_inv", ctypes.c_float),
        ("sigma", ctypes.c_float),
        ("dsigma", ctypes.c_float),
        ("c_near", ctypes.c_float),
        ("c_far", ctypes.c_float),
        ("rho0", ctypes.c_float),
        ("inv_rho0", ctypes.c_float),
        ("eos_b", ctypes.c_float),
        ("eos_gamma", ctypes.c_int),
        ("clamp_pressure", ctypes.c_int),
        ("xsph_eps", ctypes.c_float),
        ("v_max", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("use_box", ctypes.c_int),
        ("box_lo", ctypes.c_float * 3),
        ("box_hi", ctypes.c_float * 3),
    ]


class Phys64(ctypes.Structure):
    """Layout of oracle_phys_f64 (oracle/nsph_oracle.h)."""

    _fields_ = [
        ("h", ctypes.c_double),
        ("inv_h", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("dsigma", ctypes.c_double),
        ("rho0", ctypes.c_double),
        ("inv_rho0", ctypes.c_double),
        ("eos_b", ctypes.c_double),
        ("xsph_eps", ctypes.c_double),
        ("v_max", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("c_near", ctypes.c_double),
        ("c_far", ctypes.c_double),
        ("box_lo", ctypes.c_double * 3),
        ("box_hi", ctypes.c_double * 3),
        ("eos_gamma", ctypes.c_int),
        ("clamp_pressure", ctypes.c_int),
        ("use_box", ctypes.c_int),
    ]


def build(force: bool = False) -> Path:
    """Compile liboracle.so with the Makefile beside this file."""
    srcs = list(ORACLE_DIR.glob("*.c")) + list(ORACLE_DIR.glob("*.h")) + [ORACLE_DIR / "Makefile"]
    if not force and LIB_PATH.exists() and all(s.stat().st_mtime <= LIB_PATH.stat().st_mtime for s in srcs):
        return LIB_PATH
    res = subprocess.run(["make", "-B" if force else "-s", "-C", str(ORACLE_DIR)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = ctypes.CDLL(str(LIB_PATH))
    L.oracle_trunc_sat.restype = ctypes.c_int
    L.oracle_trunc_sat.argtypes = [ctypes.c_float]
    L.oracle_grid_index.restype = ctypes.c_int
    L.oracle_grid_index.argtypes = [ctypes.c_int] * 6
    L.oracle_grid_build.restype = ctypes.c_int
    L.oracle_grid_build.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    _i32p, _i32p, _i32p, _i32p]
    L.oracle_grid_query.restype = ctypes.c_longlong
    L.oracle_grid_query.argtypes = [_i32p, _i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                    _f32p, ctypes.c_float, ctypes.c_void_p, ctypes.c_longlong]
    L.oracle_sph_neighbors.restype = ctypes.c_int
    L.oracle_sph_neighbors.argtypes = [ctypes.POINTER(SphParams32), ctypes.c_int, _f32p, _i32p, _i32p, _i32p,
                                       ctypes.c_void_p, ctypes.c_void_p]
    L.oracle_sph_step_f32.restype = ctypes.c_int
    L.oracle_sph_step_f32.argtypes = [ctypes.POINTER(SphParams32), _i32p, ctypes.c_int] + [ctypes.c_void_p] * 7 + \
        [_f32p, ctypes.c_int] + [ctypes.c_void_p] * 6
    L.oracle_sph_step_f64.restype = ctypes.c_int
    L.oracle_sph_step_f64.argtypes = [ctypes.POINTER(SphParams32), ctypes.POINTER(Phys64), _i32p, ctypes.c_int] + \
        [ctypes.c_void_p] * 7 + [_f32p, ctypes.c_int] + [ctypes.c_void_p] * 6
    L.oracle_integrate_particles_f32.restype = None
    L.oracle_integrate_particles_f32.argtypes = [_f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _f32p, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_float, ctypes.c_float, _f32p, _f32p]
    L.oracle_integrate_particles_f64.restype = None
    L.oracle_integrate_particles_f64.argtypes = [_f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _f32p, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_double, ctypes.c_double, _f64p, _f64p]
    L.oracle_adj_step_f64.restype = ctypes.c_int
    L.oracle_adj_step_f64.argtypes = [ctypes.POINTER(Phys64), ctypes.c_int] + [ctypes.c_void_p] * 8 + \
        [ctypes.c_int] + [ctypes.c_void_p] * 3
    L.oracle_adj_vjp_f64.restype = ctypes.c_int
    L.oracle_adj_vjp_f64.argtypes = [ctypes.POINTER(Phys64), ctypes.c_int] + [ctypes.c_void_p] * 8 + \
        [ctypes.c_int] + [ctypes.c_void_p] * 7
    L.oracle_particle_contact_forces.restype = ctypes.c_int
    L.oracle_particle_contact_forces.argtypes = [ctypes.c_void_p, ctypes.c_float, _i32p, ctypes.c_int] + \
        [ctypes.c_void_p] * 5
    L.oracle_particle_contact_deltas.restype = ctypes.c_int
    L.oracle_particle_contact_deltas.argtypes = [ctypes.c_float, _i32p, ctypes.c_int] + [ctypes.c_void_p] * 5 + \
        [ctypes.c_float] * 5 + [ctypes.c_void_p]
    L.oracle_raycast_particles.restype = ctypes.c_int
    L.oracle_raycast_particles.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _i32p, ctypes.c_void_p,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_void_p]
    L.oracle_raycast_clamp_no_hits.restype = None
    L.oracle_raycast_clamp_no_hits.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]
    L.oracle_set_threads.restype = None
    L.oracle_set_threads.argtypes = [ctypes.c_int]
    L.oracle_get_threads.restype = ctypes.c_int
    L.oracle_get_threads.argtypes = []
    _lib = L
    return L


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def get_threads() -> int:
    return int(lib().oracle_get_threads())


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------------------
# parameter blocks from the constants dict of SPHConfig.constants()
# ---------------------------------------------------------------------------
def params32(c32: dict) -> SphParams32:
    p = SphParams32()
    for name, _ in SphParams32._fields_:
        v = c32[name]
        if name in ("box_lo", "box_hi"):
            getattr(p, name)[:] = [float(x) for x in v]
        elif isinstance(v, int):
            setattr(p, name, v)
        else:
            setattr(p, name, float(v))
    return p


def phys64(c64: dict) -> Phys64:
    p = Phys64()
    for name, _ in Phys64._fields_:
        v = c64[name]
        if name in ("box_lo", "box_hi"):
            getattr(p, name)[:] = [float(x) for x in v]
        elif isinstance(v, int):
            setattr(p, name, v)
        else:
            setattr(p, name, float(v))
    return p


# ---------------------------------------------------------------------------
# HashGrid
# ---------------------------------------------------------------------------
def grid_build(points: np.ndarray, radius: float, dims: tuple[int, int, int]) -> dict[str, np.ndarray]:
    """HashGrid.build restated: sorted cell ids, sorted point ids, ranges."""
    pts = _f32(points).reshape(-1, 3)
    n = pts.shape[0]
    nc = dims[0] * dims[1] * dims[2]
    out = {
        "point_cells": np.zeros(n, np.int32),
        "point_ids": np.zeros(n, np.int32),
        "cell_starts": np.zeros(nc, np.int32),
        "cell_ends": np.zeros(nc, np.int32),
    }
    st = lib().oracle_grid_build(pts.reshape(-1) if n else np.zeros(3, np.float32), n, float(np.float32(radius)),
                                 *dims, out["point_cells"] if n else np.zeros(1, np.int32),
                                 out["point_ids"] if n else np.zeros(1, np.int32), out["cell_starts"],
                                 out["cell_ends"])
    if st != 0:
        raise RuntimeError(f"oracle_grid_build status {st}")
    return out


def grid_query(grid: dict, dims, cell_inv: float, pos, radius: float) -> np.ndarray:
    """hash_grid_query + query_next restated: candidates in Warp order."""
    pos = _f32(pos).reshape(3)
    L = lib()
    n = L.oracle_grid_query(grid["point_ids"], grid["cell_starts"], grid["cell_ends"], *dims, float(cell_inv), pos,
                            float(radius), None, 0)
    out = np.zeros(max(n, 1), np.int32)
    L.oracle_grid_query(grid["point_ids"], grid["cell_starts"], grid["cell_ends"], *dims, float(cell_inv), pos,
                        float(radius), _p(out), n)
    return out[:n]


# ---------------------------------------------------------------------------
# SPH
# ---------------------------------------------------------------------------
def sph_neighbors(c32: dict, dims, x: np.ndarray, flags: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Neighbour lists (offsets int64 (N+1,), ids int32) in original order."""
    x = _f32(x)
    flags = _i32(flags)
    n = x.shape[0]
    p = params32(c32)
    dims_a = _i32(dims)
    counts = np.zeros(max(n, 1), np.int32)
    L = lib()
    st = L.oracle_sph_neighbors(ctypes.byref(p), n, x.reshape(-1), flags, dims_a, counts, None, None)
    if st != 0:
        raise RuntimeError(f"oracle_sph_neighbors status {st}")
    offsets = np.zeros(n + 1, np.int64)
    offsets[1:] = np.cumsum(counts[:n])
    ids = np.zeros(max(int(offsets[-1]), 1), np.int32)
    st = L.oracle_sph_neighbors(ctypes.byref(p), n, x.reshape(-1), flags, dims_a, counts, _p(offsets), _p(ids))
    if st != 0:
        raise RuntimeError(f"oracle_sph_neighbors status {st}")
    return offsets, ids[: offsets[-1]]


def sph_step(consts: dict, dims, x, v, mass, inv_mass, flags, world, gravity, f_ext=None, v_out_init=None,
             precision: str = "f64") -> dict[str, np.ndarray]:
    """One WCSPH step on the CPU (fp32 mirror or fp64 truth).

    Returns dict with x, v, rho, p, a (SPH acceleration) and a_scale
    (sum of the magnitudes of the acceleration's summands)."""
    x = _f32(x)
    v = _f32(v)
    n = x.shape[0]
    dt = np.float64 if precision == "f64" else np.float32
    out = {
        "x": np.zeros((n, 3), dt),
        "v": np.array(v_out_init if v_out_init is not None else np.zeros((n, 3)), dtype=dt),
        "rho": np.zeros(n, dt),
        "p": np.zeros(n, dt),
        "a": np.zeros((n, 3), dt),
        "a_scale": np.zeros(n, dt),
    }
    gravity = _f32(gravity).reshape(-1, 3)
    args = [
        _p(x), _p(v), _p(_f32(f_ext) if f_ext is not None else None), _p(_f32(mass)), _p(_f32(inv_mass)),
        _p(_i32(flags)), _p(_i32(world)),
        gravity.reshape(-1), gravity.shape[0],
        _p(out["x"]), _p(out["v"]), _p(out["rho"]), _p(out["p"]), _p(out["a"]), _p(out["a_scale"]),
    ]
    # keep converted temporaries alive for the call
    keep = [x, v]
    p32 = params32(consts["f32"])
    if precision == "f64":
        ph = phys64(consts["f64"])
        st = lib().oracle_sph_step_f64(ctypes.byref(p32), ctypes.byref(ph), _i32(dims), n, *args)
    else:
        st = lib().oracle_sph_step_f32(ctypes.byref(p32), _i32(dims), n, *args)
    del keep
    if st != 0:
        raise RuntimeError(f"oracle sph step status {st}")
    return out


def integrate_particles(x, v, f, inv_mass, flags, world, gravity, dt, v_max, x_new, v_new, precision="f32"):
    """integrate_particles (solver.py:10-47); x_new / v_new updated in place."""
    gravity = _f32(gravity).reshape(-1)
    args = [_f32(x).reshape(-1), _f32(v).reshape(-1), _f32(f).reshape(-1), _f32(inv_mass), _i32(flags), _i32(world),
            gravity, gravity.size // 3, _f32(x).shape[0], dt, v_max]
    if precision == "f64":
        lib().oracle_integrate_particles_f64(*args, x_new.reshape(-1), v_new.reshape(-1))
    else:
        lib().oracle_integrate_particles_f32(*args, x_new.reshape(-1), v_new.reshape(-1))


# ---------------------------------------------------------------------------
# adjoint (sph_adjoint.c): fp64 state, fp64 neighbour sets
# ---------------------------------------------------------------------------
def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class AdjScene:
    """The fixed inputs of an fp64 rollout: constants and model arrays."""

    def __init__(self, c64: dict, mass, inv_mass, flags, gravity, world=None, f_ext=None):
        self.c64 = dict(c64)
        self.mass = _f64(mass)
        self.inv_mass = _f64(inv_mass)
        self.flags = _i32(flags)
        self.n = self.mass.shape[0]
        self.world = _i32(world) if world is not None else np.zeros(self.n, np.int32)
        self.gravity = _f64(gravity).reshape(-1, 3)
        self.f_ext = _f64(f_ext) if f_ext is not None else None

    def phys(self, eos_b: float | None = None) -> Phys64:
        c = dict(self.c64)
        if eos_b is not None:
            c["eos_b"] = float(eos_b)
        return phys64(c)

    def _model_args(self):
        return [_p(self.f_ext), _p(self.mass), _p(self.inv_mass), _p(self.flags), _p(self.world), _p(self.gravity),
                self.gravity.shape[0]]


def adj_step64(scene: AdjScene, x, v, eos_b: float | None = None):
    """One fp64 step; returns (x1, v1, rho)."""
    x, v = _f64(x), _f64(v)
    n = scene.n
    xo, vo, rho = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    ph = scene.phys(eos_b)
    st = lib().oracle_adj_step_f64(ctypes.byref(ph), n, _p(x), _p(v), *scene._model_args(), _p(xo), _p(vo), _p(rho))
    if st != 0:
        raise RuntimeError(f"oracle_adj_step_f64 status {st}")
    return xo, vo, rho


def adj_vjp64(scene: AdjScene, x, v, x1_adj, v1_adj, rho_adj=None, eos_b: float | None = None):
    """Reverse of one fp64 step: (x_adj, v_adj, f_adj, b_adj)."""
    x, v = _f64(x), _f64(v)
    x1_adj, v1_adj = _f64(x1_adj), _f64(v1_adj)
    rho_adj = _f64(rho_adj) if rho_adj is not None else None
    n = scene.n
    xa, va, fa = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    ba = ctypes.c_double(0.0)
    ph = scene.phys(eos_b)
    st = lib().oracle_adj_vjp_f64(ctypes.byref(ph), n, _p(x), _p(v), *scene._model_args(), _p(x1_adj), _p(v1_adj),
                                  _p(rho_adj), _p(xa), _p(va), _p(fa), ctypes.byref(ba))
    if st != 0:
        raise RuntimeError(f"oracle_adj_vjp_f64 status {st}")
    return xa, va, fa, float(ba.value)


def rollout64(scene: AdjScene, x0, v0, steps: int, eos_b: float | None = None, keep: bool = False):
    """`steps` fp64 steps from (x0, v0). Returns (x_T, v_T) or, with keep,
    the lists of all states [x_0..x_T], [v_0..v_T]."""
    xs, vs = [_f64(x0)], [_f64(v0)]
    x, v = xs[0], vs[0]
    for _ in range(steps):
        x, v, _ = adj_step64(scene, x, v, eos_b)
        if keep:
            xs.append(x)
            vs.append(v)
    return (xs, vs) if keep else (x, v)


def mse_loss(x, target) -> float:
    """mean over particles of |x_i - y_i|^2"""
    d = _f64(x) - _f64(target)
    return float(np.sum(d * d) / d.shape[0])


def rollout_grad64(scene: AdjScene, x0, v0, steps: int, target, eos_b: float | None = None):
    """Loss mse_loss(x_T, target) and its gradient with respect to x0, v0
    and the EOS stiffness B, by reverse steps over the stored trajectory.

    Returns (loss, x0_adj, v0_adj, b_adj)."""
    xs, vs = rollout64(scene, x0, v0, steps, eos_b, keep=True)
    n = scene.n
    loss = mse_loss(xs[-1], target)
    xa = 2.0 * (xs[-1] - _f64(target)) / n
    va = np.zeros((n, 3))
    b_total = 0.0
    for t in range(steps - 1, -1, -1):
        xa, va, _, ba = adj_vjp64(scene, xs[t], vs[t], xa, va, None, eos_b)
        b_total += ba
    return loss, xa, va, b_total


# ---------------------------------------------------------------------------
# surrogate features (fp64 restatement on the fp32 neighbour lists)
# ---------------------------------------------------------------------------
def surrogate_features_py(consts: dict, dims, x, v, mass, flags):
    """The 16 dimensionless neighbour features of the surrogate step,
    restated in fp64 numpy from fp32 inputs, on the oracle's fp32 neighbour
    lists (the device's). Feature k of particle i:
      0 rho/rho0, 1 rho/rho0 - 1, 2-4 sum_j V_j W (x_j - x_i)/h,
      5-7 sum_j V_j W (v_j - v_i)/c0, 8-10 a h/c0^2, 11 sum_j V_j W r^2/h^2,
      12 V_i W(0) + sum_j V_j W, 13 sum_j V_j F (v_j - v_i).(x_i - x_j) h/c0,
      14 p/(rho0 c0^2), 15 |a| h/c0^2
    with V_j = m_j/rho_j, F = (dW/dr)/r, c0^2 = B gamma / rho0, sums over
    active neighbours j != i. Returns (features (n, 16), rho, a, dv)."""
    c32, c64 = consts["f32"], consts["f64"]
    x = _f32(x).astype(np.float64)
    v = _f32(v).astype(np.float64)
    m = _f32(mass).astype(np.float64)
    fl = _i32(flags)
    n = x.shape[0]
    off, ids = sph_neighbors(c32, dims, _f32(x), fl)
    h, sigma = c64["h"], c64["sigma"]
    counts = np.diff(off)
    ii = np.repeat(np.arange(n), counts)
    jj = ids.astype(np.int64)
    act = (fl & 1) != 0
    d = x[ii] - x[jj]
    r = np.sqrt(np.sum(d * d, axis=1))
    q = r / h
    t = 1.0 - q
    W = sigma * np.where(q <= 0.5, 6.0 * q * q * (q - 1.0) + 1.0, np.where(q < 1.0, 2.0 * t ** 3, 0.0))
    safe_r = np.where(r > 0, r, 1.0)
    F = np.where(r > 0, np.where(q <= 0.5, c64["c_near"] * (3.0 * q - 2.0), c64["c_far"] * t * t / safe_r), 0.0)
    mj = np.where(act[jj], m[jj], 0.0)
    rho = np.zeros(n)
    np.add.at(rho, ii, mj * W)
    ratio = rho / c64["rho0"]
    B, gam = c64["eos_b"], c64["eos_gamma"]
    p = np.where(rho > 0, B * (ratio ** gam - 1.0), 0.0)
    if c64["clamp_pressure"]:
        p = np.maximum(p, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        V = np.where(rho > 0, np.where(act, m, 0.0) / rho, 0.0)
        pr2 = np.where(rho > 0, p / (rho * rho), 0.0)
    nself = jj != ii
    pair = nself & act[jj] & act[ii]
    Vj, Wp, Fp = V[jj], W, F
    a = np.zeros((n, 3))
    dv = np.zeros((n, 3))
    mx = np.zeros((n, 3))
    sw = np.zeros(n)
    m2 = np.zeros(n)
    dvg = np.zeros(n)
    s = np.where(pair, mj * (pr2[ii] + pr2[jj]) * Fp, 0.0)
    rv = v[jj] - v[ii]
    c = np.where(pair, Vj * Wp, 0.0)
    for k in range(3):
        np.add.at(a[:, k], ii, -s * d[:, k])
        np.add.at(dv[:, k], ii, c * rv[:, k])
        np.add.at(mx[:, k], ii, -c * d[:, k])
    np.add.at(sw, ii, c)
    np.add.at(m2, ii, c * r * r)
    np.add.at(dvg, ii, np.where(pair, Vj * Fp * np.sum(rv * d, axis=1), 0.0))
    c0sq = float(np.float32(c32["eos_b"]) * np.float32(c32["eos_gamma"]) * np.float32(c32["inv_rho0"]))
    c0 = np.sqrt(c0sq)
    f = np.zeros((n, 16))
    f[:, 0] = ratio
    f[:, 1] = ratio - 1.0
    f[:, 2:5] = mx / h
    f[:, 5:8] = dv / c0
    f[:, 8:11] = a * h / c0sq
    f[:, 11] = m2 / (h * h)
    f[:, 12] = sw + V * sigma
    f[:, 13] = dvg * h / c0
    f[:, 14] = p / c64["rho0"] / c0sq
    f[:, 15] = np.linalg.norm(f[:, 8:11], axis=1)
    f[~act] = 0.0
    return f, rho, a, dv


# ---------------------------------------------------------------------------
# particle-particle contact (contact.c)
# ---------------------------------------------------------------------------
class ContactParams(ctypes.Structure):
    """Layout of nsph_contact_params (include/nsph.h)."""

    _fields_ = [(k, ctypes.c_float) for k in ("k_contact", "k_damp", "k_friction", "k_mu", "k_cohesion",
                                              "max_radius")]


def particle_contact_forces(x, v, radius, flags, grid_radius: float, dims, k_contact, k_damp, k_friction, k_mu,
                            k_cohesion, max_radius, f_init=None):
    """eval_particle_contact restated (fp32): forces (n, 3); rows of inactive
    particles keep f_init (zeros by default)."""
    x, v, r, fl = _f32(x), _f32(v), _f32(radius), _i32(flags)
    n = x.shape[0]
    f = np.array(f_init if f_init is not None else np.zeros((n, 3)), dtype=np.float32)
    p = ContactParams(*[float(np.float32(t)) for t in (k_contact, k_damp, k_friction, k_mu, k_cohesion, max_radius)])
    st = lib().oracle_particle_contact_forces(ctypes.byref(p), float(np.float32(grid_radius)), _i32(dims), n, _p(x),
                                              _p(v), _p(r), _p(fl), _p(f))
    if st != 0:
        raise RuntimeError(f"oracle_particle_contact_forces status {st}")
    return f


def particle_contact_deltas(x, v, inv_mass, radius, flags, grid_radius: float, dims, k_mu, k_cohesion, max_radius,
                            dt, relaxation, deltas_init=None):
    """solve_particle_particle_contacts restated (fp32): deltas_init + corrections."""
    x, v, w, r, fl = _f32(x), _f32(v), _f32(inv_mass), _f32(radius), _i32(flags)
    n = x.shape[0]
    d = np.array(deltas_init if deltas_init is not None else np.zeros((n, 3)), dtype=np.float32)
    st = lib().oracle_particle_contact_deltas(float(np.float32(grid_radius)), _i32(dims), n, _p(x), _p(v), _p(w),
                                              _p(r), _p(fl), *[float(np.float32(t)) for t in
                                                               (k_mu, k_cohesion, max_radius, dt, relaxation)],
                                              _p(d))
    if st != 0:
        raise RuntimeError(f"oracle_particle_contact_deltas status {st}")
    return d


# ---------------------------------------------------------------------------
# particle raycast depth camera (raycast.c)
# ---------------------------------------------------------------------------
class RaycastCamera(ctypes.Structure):
    """Layout of nsph_raycast_camera (include/nsph.h)."""

    _fields_ = [("position", ctypes.c_float * 3), ("direction", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("right", ctypes.c_float * 3), ("fov_scale", ctypes.c_float), ("aspect_ratio", ctypes.c_float),
                ("width", ctypes.c_int), ("height", ctypes.c_int), ("max_distance", ctypes.c_float)]


def raycast_camera(position, direction, up, right, fov_scale, aspect_ratio, width, height, max_distance):
    c = RaycastCamera()
    for name, v in (("position", position), ("direction", direction), ("up", up), ("right", right)):
        getattr(c, name)[:] = [float(np.float32(t)) for t in v]
    c.fov_scale, c.aspect_ratio = float(np.float32(fov_scale)), float(np.float32(aspect_ratio))
    c.width, c.height, c.max_distance = int(width), int(height), float(np.float32(max_distance))
    return c


def raycast_particles(x, radius, dims, cam: RaycastCamera, search_radius, march_step, max_steps, depth_init=None,
                      clamp=True):
    """The particle path of SensorRaycast.update restated (fp32): depth
    (height, width) from depth_init (max_distance everywhere by default),
    then the no-hit clamp to -1 when `clamp`."""
    x, r = _f32(x), _f32(radius)
    n = x.shape[0]
    depth = np.array(depth_init if depth_init is not None else
                     np.full((cam.height, cam.width), cam.max_distance), dtype=np.float32)
    st = lib().oracle_raycast_particles(_p(x), _p(r), n, _i32(dims), ctypes.byref(cam),
                                        float(np.float32(search_radius)), float(np.float32(march_step)),
                                        int(max_steps), _p(depth))
    if st != 0:
        raise RuntimeError(f"oracle_raycast_particles status {st}")
    if clamp:
        lib().oracle_raycast_clamp_no_hits(_p(depth), depth.size, cam.max_distance)
    return depth


def raycast_particles_py(x, radius, dims, cam: RaycastCamera, search_radius, march_step, max_steps):
    """The same loop in pure Python with numpy float32 scalars (small cases):
    a check of raycast.c. Returns the clamped depth image."""
    f = np.float32
    x, radius = np.asarray(x, np.float32), np.asarray(radius, np.float32)
    grid = grid_build_py(x, search_radius, dims)
    inv = f(1.0) / f(search_radius)

    def dot(a, b):
        return f(f(f(a[0] * b[0]) + f(a[1] * b[1])) + f(a[2] * b[2]))

    def query(p, rad):
        out = []
        lo, hi = [], []
        for a in range(3):
            s0 = trunc_sat_py(f(f(p[a] - f(rad)) * inv))
            e0 = trunc_sat_py(f(f(p[a] + f(rad)) * inv))
            e0 = min(e0, s0 + dims[a] - 1)
            lo.append(s0)
            hi.append(max(e0, s0))
        for z in range(lo[2], hi[2] + 1):
            for y in range(lo[1], hi[1] + 1):
                for xx in range(lo[0], hi[0] + 1):
                    c = [max(v + (1 << 20), 0) % dims[a] for a, v in enumerate((xx, y, z))]
                    cell = c[2] * dims[0] * dims[1] + c[1] * dims[0] + c[0]
                    out.extend(grid["point_ids"][grid["cell_starts"][cell]:grid["cell_ends"][cell]].tolist())
        return out

    w, h = cam.width, cam.height
    maxd = f(cam.max_distance)
    depth = np.full((h, w), maxd, np.float32)
    o = [f(v) for v in cam.position]
    for py in range(h):
        for px in range(w):
            ndc_x = f(f(f(f(2.0) * f(px)) + f(1.0)) / f(w)) - f(1.0)
            ndc_y = f(1.0) - f(f(f(f(2.0) * f(py)) + f(1.0)) / f(h))
            cx = f(f(ndc_x * f(cam.fov_scale)) * f(cam.aspect_ratio))
            cy = f(ndc_y * f(cam.fov_scale))
            d = [f(f(f(cam.right[k]) * cx) + f(f(cam.up[k]) * cy)) + f(cam.direction[k]) for k in range(3)]
            d = [f(v) for v in d]
            ln = f(np.sqrt(dot(d, d)))
            d = [f(v / ln) if ln > 0 else f(0.0) for v in d]
            best = depth[py, px]
            if best < 0:
                best = maxd
            s, t = 0, f(0.0)
            while s < max_steps and t <= maxd and t <= best:
                p = [f(o[k] + f(d[k] * t)) for k in range(3)]
                for j in query(p, search_radius):
                    rad = radius[j]
                    if rad <= 0:
                        continue
                    oc = [f(o[k] - x[j, k]) for k in range(3)]
                    proj = dot(d, oc)
                    cc = f(dot(oc, oc) - f(rad * rad))
                    disc = f(f(proj * proj) - cc)
                    if disc < 0:
                        continue
                    sq = f(np.sqrt(disc))
                    th = f(-proj - sq)
                    if th < 0:
                        th = f(-proj + sq)
                    if th < 0 or th > maxd:
                        continue
                    if th < best:
                        best = th
                        depth[py, px] = th
                s += 1
                t = f(t + f(march_step))
    depth[depth >= maxd] = f(-1.0)
    return depth


# ---------------------------------------------------------------------------
# pure-Python restatements (small cases; checks of the C oracle)
# ---------------------------------------------------------------------------
def trunc_sat_py(v: np.float32) -> int:
    v = float(v)
    if math.isnan(v):
        return 0
    if v >= 2147483648.0:
        return 2**31 - 1
    if v <= -2147483648.0:
        return -(2**31)
    return int(math.trunc(v))


def cell_of_py(p, inv: np.float32, dims) -> int:
    """Warp hash_grid_index of point p (fp32 products)."""
    c = []
    for a in range(3):
        vc = trunc_sat_py(np.float32(np.float32(p[a]) * inv)) + (1 << 20)
        c.append(max(vc, 0) % dims[a])
    return c[2] * dims[0] * dims[1] + c[1] * dims[0] + c[0]


def grid_build_py(points, radius, dims):
    """HashGrid.build with Python sorting (stable sort by cell id)."""
    inv = np.float32(1.0) / np.float32(radius)
    keys = [cell_of_py(p, inv, dims) for p in np.asarray(points, np.float32)]
    order = sorted(range(len(keys)), key=lambda i: keys[i])  # Python's sort is stable
    nc = dims[0] * dims[1] * dims[2]
    starts = np.zeros(nc, np.int32)
    ends = np.zeros(nc, np.int32)
    cells = [keys[i] for i in order]
    for k, c in enumerate(cells):
        if k == 0 or cells[k - 1] != c:
            starts[c] = k
        if k == len(cells) - 1 or cells[k + 1] != c:
            ends[c] = k + 1
    return {"point_cells": np.array(cells, np.int32), "point_ids": np.array(order, np.int32),
            "cell_starts": starts, "cell_ends": ends}


def neighbors_brute_py(x, h2: np.float32, flags):
    """All j with fp32 r2 = fma(dz,dz,fma(dy,dy,dx*dx)) < h2 (O(N^2), as a set
    per particle): the grid-free definition of the neighbour set."""
    x = np.asarray(x, np.float32)
    n = len(x)
    d = x[:, None, :] - x[None, :, :]
    # numpy has no fma; emulate exactly through float64 (exact products of
    # fp32 values, one rounding per fma)
    dx, dy, dz = (d[..., k].astype(np.float64) for k in range(3))
    t = (dx * dx).astype(np.float32).astype(np.float64)
    t = (dy * dy + t).astype(np.float32).astype(np.float64)
    r2 = (dz * dz + t).astype(np.float32)
    act = (np.asarray(flags) & 1) != 0
    out = []
    for i in range(n):
        out.append(set(np.nonzero((r2[i] < h2) & act)[0].tolist()) if act[i] else set())
    return out


def lattice_py(pos, vel, dim_x, dim_y, dim_z, cell_x, cell_y, cell_z, jitter, seed_base=0):
    """add_particle_grid's positions (builder.py:8085-8096) with explicit
    loops: index = iy*(dim_x*dim_z) + ix*dim_z + iz, identity rotation, then
    jitter from default_rng(42 + seed_base) over the (N, 3) array."""
    pts = []
    for iy in range(dim_y):
        for ix in range(dim_x):
            for iz in range(dim_z):
                pts.append([ix * cell_x + pos[0], iy * cell_y + pos[1], iz * cell_z + pos[2]])
    pts = np.array(pts, dtype=np.float64)
    rng = np.random.default_rng(42 + seed_base)
    pts += (rng.random(pts.shape) - 0.5) * jitter
    return pts


def cubic_spline_py(r: float, h: float) -> float:
    """W(r) of the 3-D cubic spline with support h (Monaghan 1992)."""
    q = r / h
    s = 8.0 / (math.pi * h**3)
    if q <= 0.5:
        return s * (6.0 * (q**3 - q**2) + 1.0)
    if q < 1.0:
        return s * 2.0 * (1.0 - q) ** 3
    return 0.0


# ---------------------------------------------------------------------------
# particles against static analytic shapes; the XPBD particle update (shapes.c)
# ---------------------------------------------------------------------------
class Shape(ctypes.Structure):
    """Layout of nsph_shape (include/nsph.h)."""

    _fields_ = [("type", ctypes.c_int), ("flags", ctypes.c_int), ("world", ctypes.c_int), ("reserved", ctypes.c_int),
                ("pos", ctypes.c_float * 3), ("rot", ctypes.c_float * 4), ("scale", ctypes.c_float * 3),
                ("ke", ctypes.c_float), ("kd", ctypes.c_float), ("kf", ctypes.c_float), ("mu", ctypes.c_float)]


class SoftContactParams(ctypes.Structure):
    """Layout of nsph_soft_contact_params (include/nsph.h)."""

    _fields_ = [(k, ctypes.c_float) for k in ("ke", "kd", "kf", "mu", "adhesion", "restitution", "relaxation", "dt")]


def shapes_array(shapes) -> ctypes.Array:
    """ctypes array of Shape from dicts with the nsph_shape field names."""
    arr = (Shape * max(1, len(shapes)))()
    for i, s in enumerate(shapes):
        arr[i].type = int(s["type"])
        arr[i].flags = int(s.get("flags", 1 << 2))
        arr[i].world = int(s.get("world", -1))
        arr[i].pos[:] = [float(np.float32(t)) for t in s.get("pos", (0.0, 0.0, 0.0))]
        arr[i].rot[:] = [float(np.float32(t)) for t in s.get("rot", (0.0, 0.0, 0.0, 1.0))]
        arr[i].scale[:] = [float(np.float32(t)) for t in s.get("scale", (0.0, 0.0, 0.0))]
        for k in ("ke", "kd", "kf", "mu"):
            setattr(arr[i], k, float(np.float32(s.get(k, 0.0))))
    return arr


def soft_contact_params(ke, kd, kf, mu, adhesion, restitution, relaxation, dt) -> SoftContactParams:
    return SoftContactParams(*[float(np.float32(t)) for t in (ke, kd, kf, mu, adhesion, restitution, relaxation, dt)])


def _shape_lib():
    L = lib()
    if not getattr(L, "_shapes_declared", False):
        L.oracle_soft_contacts_create.restype = ctypes.c_int
        L.oracle_soft_contacts_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_void_p] * 4 + [ctypes.c_float, ctypes.c_int] + [ctypes.c_void_p] * 6
        L.oracle_shape_contact_forces.restype = ctypes.c_int
        L.oracle_shape_contact_forces.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 11
        L.oracle_shape_contact_deltas.restype = ctypes.c_int
        L.oracle_shape_contact_deltas.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 12
        L.oracle_shape_restitution.restype = ctypes.c_int
        L.oracle_shape_restitution.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 10
        L.oracle_apply_particle_deltas.restype = None
        L.oracle_apply_particle_deltas.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + \
            [ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
        L._shapes_declared = True
    return L


def soft_contacts_create(shapes, x, radius, flags, world=None, margin=0.01, max_contacts=None) -> dict:
    """create_soft_contacts restated: contacts in (particle, shape) order."""
    arr = shapes if isinstance(shapes, ctypes.Array) else shapes_array(shapes)
    ns = len(shapes)
    x, r, fl = _f32(x), _f32(radius), _i32(flags)
    n = x.shape[0]
    mx = n * ns if max_contacts is None else int(max_contacts)
    out = {"count": np.zeros(1, np.int32), "particle": np.zeros(max(mx, 1), np.int32),
           "shape": np.zeros(max(mx, 1), np.int32), "body_pos": np.zeros((max(mx, 1), 3), np.float32),
           "body_vel": np.zeros((max(mx, 1), 3), np.float32), "normal": np.zeros((max(mx, 1), 3), np.float32)}
    w = _i32(world) if world is not None else None
    st = _shape_lib().oracle_soft_contacts_create(
        ctypes.cast(arr, ctypes.c_void_p), ns, n, _p(x), _p(r), _p(fl), _p(w), float(np.float32(margin)), mx,
        _p(out["count"]), _p(out["particle"]), _p(out["shape"]), _p(out["body_pos"]), _p(out["body_vel"]),
        _p(out["normal"]))
    if st != 0:
        raise RuntimeError(f"oracle_soft_contacts_create status {st}")
    out["max"] = mx
    out["n"] = int(min(mx, out["count"][0]))
    return out


def _contact_args(c):
    return [_p(c["particle"]), _p(c["shape"]), _p(c["body_pos"]), _p(c["body_vel"]), _p(c["normal"])]


def shape_contact_forces(shapes, contacts, prm, x, v, radius, flags, f) -> np.ndarray:
    """eval_particle_body_contact restated: returns f minus the contact forces."""
    arr = shapes if isinstance(shapes, ctypes.Array) else shapes_array(shapes)
    f = np.array(f, dtype=np.float32)
    st = _shape_lib().oracle_shape_contact_forces(
        ctypes.cast(arr, ctypes.c_void_p), contacts["n"], *_contact_args(contacts), ctypes.byref(prm), _p(_f32(x)),
        _p(_f32(v)), _p(_f32(radius)), _p(_i32(flags)), _p(f))
    if st != 0:
        raise RuntimeError(f"oracle_shape_contact_forces status {st}")
    return f


def shape_contact_deltas(shapes, contacts, prm, x, v, inv_mass, radius, flags, delta) -> np.ndarray:
    """solve_particle_shape_contacts restated: returns delta plus the corrections."""
    arr = shapes if isinstance(shapes, ctypes.Array) else shapes_array(shapes)
    d = np.array(delta, dtype=np.float32)
    st = _shape_lib().oracle_shape_contact_deltas(
        ctypes.cast(arr, ctypes.c_void_p), contacts["n"], *_contact_args(contacts), ctypes.byref(prm), _p(_f32(x)),
        _p(_f32(v)), _p(_f32(inv_mass)), _p(_f32(radius)), _p(_i32(flags)), _p(d))
    if st != 0:
        raise RuntimeError(f"oracle_shape_contact_deltas status {st}")
    return d


def shape_restitution(contacts, prm, v_new, x_old, v_old, radius, flags, v_out) -> np.ndarray:
    """apply_particle_shape_restitution restated: returns v_out plus the updates."""
    vo = np.array(v_out, dtype=np.float32)
    vn = _f32(v_new)
    st = _shape_lib().oracle_shape_restitution(
        vn.shape[0], contacts["n"], _p(contacts["particle"]), _p(contacts["body_pos"]), _p(contacts["body_vel"]),
        _p(contacts["normal"]), ctypes.byref(prm), _p(vn), _p(_f32(x_old)), _p(_f32(v_old)), _p(_f32(radius)),
        _p(_i32(flags)), _p(vo))
    if st != 0:
        raise RuntimeError(f"oracle_shape_restitution status {st}")
    return vo


def apply_particle_deltas(x_orig, x_pred, flags, delta, dt, v_max, x_out, v_out):
    """apply_particle_deltas restated; x_out / v_out updated in place (active rows)."""
    _shape_lib().oracle_apply_particle_deltas(_f32(x_orig).shape[0], _p(_f32(x_orig)), _p(_f32(x_pred)),
                                              _p(_i32(flags)), _p(_f32(delta)), float(np.float32(dt)),
                                              float(np.float32(v_max)), _p(x_out), _p(v_out))


def xpbd_particle_step(m: dict, x_in, v_in, f_in, dt: float, iterations: int, relaxation: float,
                       contacts=None, enable_restitution: bool = False, dims=(128, 128, 128), x_out_init=None,
                       v_out_init=None):
    """SolverXPBD.step for a particle model with static shapes
    (newton/_src/solvers/xpbd/solver_xpbd.py:260-319, 362-440, 504, 638-714),
    restated on the oracle's kernels, including the reference's buffer
    ping-pong between the input and output states (_apply_particle_deltas,
    :157-197).

    m: dict of model arrays and scalars (inv_mass, radius, flags, world,
    gravity, v_max, particle_mu, particle_cohesion, max_radius, shapes,
    soft: the nsph_soft_contact_params values except relaxation and dt).
    x_out_init / v_out_init: the output state's buffers before the step
    (rows the step does not write keep them; zeros by default).
    Returns (x_in_after, v_in_after, x_out, v_out): the reference also
    writes intermediate iterates into the input state's buffers."""
    n = x_in.shape[0]
    xi, vi = np.array(x_in, np.float32), np.array(v_in, np.float32)
    xo = np.array(x_out_init, np.float32) if x_out_init is not None else np.zeros_like(xi)
    vo = np.array(v_out_init, np.float32) if v_out_init is not None else np.zeros_like(vi)
    q_init, qd_init = xi.copy(), vi.copy()
    integrate_particles(xi, vi, f_in, m["inv_mass"], m["flags"], m["world"], m["gravity"], dt, m["v_max"], xo, vo)
    grid_r = float(np.float32(m["max_radius"] * 2.0 + m["particle_cohesion"]))
    use_pp = n > 1 and m["max_radius"] > 0.0
    prm = soft_contact_params(*m["soft"][:6], relaxation, dt)
    bufs = {"in": (xi, vi), "out": (xo, vo)}
    cur = "out"
    counter = 0
    grid_x = xo.copy()  # the grid is built once, on the predicted positions
    for _ in range(iterations):
        xq, vq = bufs[cur]
        d = np.zeros((n, 3), np.float32)
        if contacts is not None and len(m["shapes"]):
            d = shape_contact_deltas(m["shapes"], contacts, prm, xq, vq, m["inv_mass"], m["radius"], m["flags"], d)
        if use_pp:
            d = particle_contact_deltas_on_grid(grid_x, xq, vq, m["inv_mass"], m["radius"], m["flags"], grid_r, dims,
                                                m["particle_mu"], m["particle_cohesion"], m["max_radius"], dt,
                                                relaxation, d)
        # reference ping-pong: iteration 0 reads the output state and writes the input state's buffers
        if counter == 0:
            src, dst = "out", "in"
        else:
            src, dst = "in", "out"
        counter = 1 - counter
        apply_particle_deltas(q_init, bufs[src][0], m["flags"], d, dt, m["v_max"], bufs[dst][0], bufs[dst][1])
        cur = dst
    if cur != "out":
        xo[...] = bufs[cur][0]
        vo[...] = bufs[cur][1]
    if enable_restitution and contacts is not None:
        vo[...] = shape_restitution(contacts, prm, vo.copy(), q_init, qd_init, m["radius"], m["flags"], vo)
    return xi, vi, xo, vo


def particle_contact_deltas_on_grid(grid_x, x, v, inv_mass, radius, flags, grid_radius, dims, k_mu, k_cohesion,
                                    max_radius, dt, relaxation, deltas_init):
    """solve_particle_particle_contacts with the grid built on grid_x and the
    particles at x (the XPBD iterations keep the grid of the predicted
    positions while the particles move)."""
    L = _shape_lib()
    if not getattr(L, "_deltas_grid_declared", False):
        L.oracle_particle_contact_deltas_grid.restype = ctypes.c_int
        L.oracle_particle_contact_deltas_grid.argtypes = [ctypes.c_void_p, ctypes.c_float, _i32p, ctypes.c_int] + \
            [ctypes.c_void_p] * 5 + [ctypes.c_float] * 5 + [ctypes.c_void_p]
        L._deltas_grid_declared = True
    gx, x32, v32 = _f32(grid_x), _f32(x), _f32(v)
    w, r, fl = _f32(inv_mass), _f32(radius), _i32(flags)
    d = np.array(deltas_init, dtype=np.float32)
    st = L.oracle_particle_contact_deltas_grid(_p(gx), float(np.float32(grid_radius)), _i32(dims), x32.shape[0],
                                               _p(x32), _p(v32), _p(w), _p(r), _p(fl),
                                               *[float(np.float32(t)) for t in
                                                 (k_mu, k_cohesion, max_radius, dt, relaxation)], _p(d))
    if st != 0:
        raise RuntimeError(f"oracle_particle_contact_deltas_grid status {st}")
    return d
