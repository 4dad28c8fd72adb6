"""State dumps, trajectory recording and JSONL metrics.

The reference serialises a model and its state history through its
``ViewerFile`` recorder (newton/_src/viewer/viewer_file.py:1021-1233, json /
cbor2, a HashGrid written as None) and copies states with ``State.assign``;
it has no solver checkpoint. Here:

- ``save_state`` / ``load_state``: one state (positions, velocities, forces
  and every namespaced array such as ``sph.density``) to and from an ``.npz``
  file, so that a run can stop and resume from the same arrays;
- ``TrajectoryRecorder``: every k-th state of a run into one ``.npz`` (frames
  stacked along axis 0), e.g. for surrogate training data or offline
  analysis;
- ``MetricsLog``: one JSON object per line (particle-steps/s, density error,
  fallback counts and the like), appended and flushed as it goes.

A HashGrid is not saved: the solvers rebuild it from the positions at every
step.
"""

from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np
import torch

from .sim.state import AttributeNamespace, State

_FORMAT = "newton_sph_dev_b200.state/1"


def _npz(path: Path) -> Path:
    """The name numpy writes for ``path`` (it appends .npz when missing)."""
    return path if path.suffix == ".npz" else path.with_name(path.name + ".npz")


def _state_arrays(state: State) -> dict[str, torch.Tensor]:
    """Every tensor of the state, namespaced ones as 'ns.name'."""
    out = {}
    for k, v in vars(state).items():
        if k.startswith("_"):
            continue
        if isinstance(v, torch.Tensor):
            out[k] = v
        elif isinstance(v, AttributeNamespace):
            for kk, vv in vars(v).items():
                if not kk.startswith("_") and isinstance(vv, torch.Tensor):
                    out[f"{k}.{kk}"] = vv
    return out


def save_state(path, state: State, step: int | None = None, sim_time: float | None = None, **meta) -> Path:
    """Write the state's arrays to ``path`` (``.npz``), with the step index,
    the simulated time and any extra JSON-serialisable metadata."""
    path = Path(path)
    arrays = {k: v.detach().cpu().numpy() for k, v in _state_arrays(state).items()}
    info = {"format": _FORMAT, "step": step, "sim_time": sim_time, "arrays": sorted(arrays), **meta}
    np.savez(path, __meta__=np.array(json.dumps(info)), **arrays)
    return _npz(path)


def read_state_file(path) -> tuple[dict[str, np.ndarray], dict]:
    """The arrays and the metadata of a file written by ``save_state``."""
    with np.load(path, allow_pickle=False) as d:
        info = json.loads(str(d["__meta__"]))
        if info.get("format") != _FORMAT:
            raise ValueError(f"{path}: not a state file ({info.get('format')!r})")
        arrays = {k: d[k] for k in info["arrays"]}
    return arrays, info


def load_state(path, state: State, strict: bool = True) -> dict:
    """Copy the arrays of a file written by ``save_state`` into an existing
    state (on its device). Returns the file's metadata.

    Raises:
        ValueError: an array's shape or dtype differs from the state's, or
            (strict) the file and the state do not hold the same arrays.
    """
    arrays, info = read_state_file(path)
    have = _state_arrays(state)
    if strict and set(arrays) != set(have):
        raise ValueError(f"{path}: arrays {sorted(arrays)} do not match the state's {sorted(have)}")
    for k, a in arrays.items():
        t = have.get(k)
        if t is None:
            continue
        if tuple(a.shape) != tuple(t.shape) or str(a.dtype) != str(t.dtype).replace("torch.", ""):
            raise ValueError(f"{path}: '{k}' is {a.dtype}{a.shape}, the state's is {t.dtype}{tuple(t.shape)}")
        with torch.no_grad():
            t.copy_(torch.from_numpy(a))
    return info


class TrajectoryRecorder:
    """Every ``every``-th recorded state of a run, written to one ``.npz``.

    ``record(state, step)`` copies the chosen arrays to host memory (a
    synchronising copy); ``save()`` stacks the frames along axis 0 together
    with their step indices. ``max_frames`` bounds the host memory held.
    """

    def __init__(self, path, every: int = 1, arrays=("particle_q", "particle_qd"), max_frames: int | None = None):
        if every < 1:
            raise ValueError("every must be at least 1")
        self.path = Path(path)
        self.every = int(every)
        self.arrays = tuple(arrays)
        self.max_frames = max_frames
        self.frames: dict[str, list[np.ndarray]] = {k: [] for k in self.arrays}
        self.steps: list[int] = []
        self._calls = 0

    def record(self, state: State, step: int | None = None) -> bool:
        """Record the state if this call is one of every ``every``; returns
        whether it was recorded."""
        call = self._calls
        self._calls += 1
        if call % self.every:
            return False
        if self.max_frames is not None and len(self.steps) >= self.max_frames:
            raise RuntimeError(f"trajectory holds {self.max_frames} frames already")
        have = _state_arrays(state)
        for k in self.arrays:
            if k not in have:
                raise KeyError(f"state has no array '{k}'")
            self.frames[k].append(have[k].detach().cpu().numpy().copy())
        self.steps.append(call if step is None else int(step))
        return True

    def __len__(self) -> int:
        return len(self.steps)

    def save(self, **meta) -> Path:
        """Write the recorded frames; returns the path."""
        out = {k.replace(".", "__"): np.stack(v) if v else np.zeros((0,)) for k, v in self.frames.items()}
        info = {"format": "newton_sph_dev_b200.trajectory/1", "every": self.every, "arrays": list(self.arrays),
                **meta}
        np.savez(self.path, __meta__=np.array(json.dumps(info)), steps=np.asarray(self.steps, np.int64), **out)
        return _npz(self.path)

    @staticmethod
    def load(path) -> tuple[dict[str, np.ndarray], np.ndarray, dict]:
        """The frames (name -> array of shape (frames, ...)), step indices and
        metadata of a saved trajectory."""
        with np.load(path, allow_pickle=False) as d:
            info = json.loads(str(d["__meta__"]))
            frames = {k: d[k.replace(".", "__")] for k in info["arrays"]}
            steps = d["steps"]
        return frames, steps, info


class MetricsLog:
    """Append-only JSON-lines metrics: ``log(step=..., rate=..., ...)``
    writes one object per line with a wall-clock timestamp and flushes it."""

    def __init__(self, path, mode: str = "a"):
        self.path = Path(path)
        self._f = open(self.path, mode, encoding="utf-8")

    def log(self, **fields) -> dict:
        rec = {"time": time.time(), **{k: _jsonable(v) for k, v in fields.items()}}
        self._f.write(json.dumps(rec) + "\n")
        self._f.flush()
        return rec

    def close(self) -> None:
        if not self._f.closed:
            self._f.close()

    def __enter__(self) -> "MetricsLog":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    @staticmethod
    def read(path) -> list[dict]:
        with open(path, encoding="utf-8") as f:
            return [json.loads(line) for line in f if line.strip()]


def _jsonable(v):
    if isinstance(v, torch.Tensor):
        v = v.detach().cpu()
        return v.item() if v.numel() == 1 else v.tolist()
    if isinstance(v, np.generic):
        return v.item()
    if isinstance(v, np.ndarray):
        return v.tolist()
    return v


__all__ = ["MetricsLog", "TrajectoryRecorder", "load_state", "read_state_file", "save_state"]
