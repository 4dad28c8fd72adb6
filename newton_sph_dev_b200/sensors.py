"""Raycast depth camera over the particles, on this library's HashGrid.

:class:`SensorRaycast` mirrors the reference's class of the same name
(newton/_src/sensors/sensor_raycast.py:31-481): the same constructor, camera
basis, ``update``, depth-image accessors and camera setters, with depth values
> 0 for a hit and -1 for none. Its particle path
(``update(state, include_particles=True)``, sensor_raycast.py:185-263,
272-320) runs in libnsph.so: a HashGrid(128, 128, 128) built on the particle
positions with the cell width max radius + 1e-6, then
``nsph_raycast_particles`` (the march of sensor_raycast_particles_kernel,
newton/_src/geometry/raycast.py:1090-1180) and ``nsph_raycast_clamp_no_hits``.

The reference also intersects the model's collision shapes; this package has
no shape pipeline, so a model that carries shapes is refused.
"""

from __future__ import annotations

import ctypes
import math
import warnings

import numpy as np
import torch

from . import _lib
from .hashgrid import HashGrid

INT32_MAX = (1 << 31) - 1
# upper bound on the march samples of one pixel (the reference's limit)
MAX_PARTICLE_RAY_MARCH_STEPS = 1 << 20

DEPRECATION_MESSAGE = ("SensorRaycast is deprecated; use SensorTiledCamera instead. "
                       "See the SensorRaycast class docstring for a migration example.")


def camera_basis(direction, up) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Orthonormal (direction, up, right) from a view direction and an up
    hint, as SensorRaycast._compute_camera_basis (sensor_raycast.py:157-183):
    right = direction x up (another up hint when they are parallel), then up
    = right x direction, all normalised."""
    direction = np.asarray(direction, dtype=np.float32)
    up = np.asarray(up, dtype=np.float32)
    d = direction / np.linalg.norm(direction)
    u = up / np.linalg.norm(up)
    r = np.cross(d, u)
    rn = np.linalg.norm(r)
    if rn < 1e-8:
        temp_up = np.array([0.0, 0.0, 1.0], dtype=np.float32) if abs(d[2]) < 0.9 else \
            np.array([0.0, 1.0, 0.0], dtype=np.float32)
        r = np.cross(d, temp_up)
        rn = np.linalg.norm(r)
    r = r / rn
    u = np.cross(r, d)
    u = u / np.linalg.norm(u)
    return d, u, r


def march_steps(max_distance: float, step: float) -> tuple[int, bool, float]:
    """(steps, truncated, requested): samples needed to march max_distance in
    steps of `step`, capped at MAX_PARTICLE_RAY_MARCH_STEPS
    (sensor_raycast.py:342-361)."""
    if step <= 0.0:
        raise ValueError("particle march step must be positive.")
    ratio = float(max_distance) / float(step)
    if ratio <= 0.0:
        return 1, False, 1.0
    max_allowed = min(INT32_MAX, MAX_PARTICLE_RAY_MARCH_STEPS)
    if not math.isfinite(ratio):
        return max_allowed, True, math.inf
    requested = math.floor(ratio) + 1
    if requested > max_allowed:
        return max_allowed, True, requested
    return int(requested), False, int(requested)


class SensorRaycast:
    """Depth camera: one ray per pixel through the pixel centre, perspective
    projection with vertical field of view ``fov_radians``; depth is the
    distance to the nearest particle sphere along the ray, -1 where none is
    hit within ``max_distance``."""

    def __init__(self, model, camera_position, camera_direction, camera_up, fov_radians: float, width: int,
                 height: int, *, max_distance: float = 1000.0):
        warnings.warn(DEPRECATION_MESSAGE, DeprecationWarning, stacklevel=2)
        if int(getattr(model, "shape_count", 0) or 0) > 0:
            raise NotImplementedError("the sensor raycasts particles only: shape raycasts (the model has "
                                      f"{model.shape_count} shapes) are not provided by this package")
        self.model = model
        self.device = model.device
        self.width = int(width)
        self.height = int(height)
        self.fov_radians = fov_radians
        self.aspect_ratio = float(width) / float(height)
        self.max_distance = max_distance
        self.camera_position = np.array(camera_position, dtype=np.float32)
        self.fov_scale = math.tan(fov_radians * 0.5)
        self._depth_buffer = torch.zeros((self.height, self.width), dtype=torch.float32, device=self.device)
        self.depth_image = self._depth_buffer
        self._compute_camera_basis(np.array(camera_direction, dtype=np.float32),
                                   np.array(camera_up, dtype=np.float32))
        self._particle_grid: HashGrid | None = None
        self._particle_step_warning_emitted = False

    def _compute_camera_basis(self, direction: np.ndarray, up: np.ndarray) -> None:
        self.camera_direction, self.camera_up, self.camera_right = camera_basis(direction, up)

    def _camera(self) -> _lib.NsphRaycastCamera:
        c = _lib.NsphRaycastCamera()
        c.position[:] = [float(v) for v in self.camera_position]
        c.direction[:] = [float(v) for v in self.camera_direction]
        c.up[:] = [float(v) for v in self.camera_up]
        c.right[:] = [float(v) for v in self.camera_right]
        c.fov_scale = float(self.fov_scale)
        c.aspect_ratio = float(self.aspect_ratio)
        c.width, c.height = self.width, self.height
        c.max_distance = float(self.max_distance)
        return c

    def update(self, state, *, include_particles: bool = False, particle_march_step: float | None = None) -> None:
        """Render the depth image of ``state``. Particles count only with
        include_particles (as in the reference, off by default);
        particle_march_step defaults to half of max radius + 1e-6."""
        if include_particles and particle_march_step is not None and particle_march_step <= 0.0:
            raise ValueError("particle_march_step must be positive when provided.")
        self._depth_buffer.fill_(self.max_distance)
        if include_particles and self._does_state_have_particles(state):
            self._raycast_particles(state, particle_march_step)
        self._clamp_no_hits()

    def _does_state_have_particles(self, state) -> bool:
        if state.particle_q is None or state.particle_count == 0:
            return False
        if self.model.particle_radius is None or self.model.particle_max_radius <= 0.0:
            raise ValueError("Model must have valid particle radius to raycast when particles are present.")
        return True

    def _get_particle_grid(self) -> HashGrid:
        if self._particle_grid is None:
            self._particle_grid = HashGrid(128, 128, 128, device=self.device)
        return self._particle_grid

    def _compute_particle_march_steps(self, step: float) -> tuple[int, bool, float]:
        return march_steps(self.max_distance, step)

    def _raycast_particles(self, state, march_step: float | None) -> None:
        n = state.particle_count
        search_radius = float(self.model.particle_max_radius) + 1.0e-6
        step = march_step if march_step is not None else 0.5 * search_radius
        max_steps, truncated, requested = self._compute_particle_march_steps(step)
        if truncated and not self._particle_step_warning_emitted:
            requested_msg = "infinite" if not math.isfinite(requested) else f"{requested:,}"
            max_allowed = min(INT32_MAX, MAX_PARTICLE_RAY_MARCH_STEPS)
            warnings.warn(f"Particle ray marching limited to {max_allowed:,} steps (requested {requested_msg}). "
                          "Increase particle_march_step or reduce max_distance for full coverage.",
                          RuntimeWarning, stacklevel=3)
            self._particle_step_warning_emitted = True
        x = state.particle_q
        radius = self.model.particle_radius
        for t, name, shape in ((x, "particle_q", (n, 3)), (radius, "particle_radius", (n,))):
            if t.dtype != torch.float32 or tuple(t.shape) != shape or not t.is_contiguous() or not t.is_cuda:
                raise ValueError(f"{name} must be a contiguous CUDA float32 tensor of shape {shape}")
        grid = self._get_particle_grid()
        grid.reserve(n)
        grid.build(x, search_radius)
        cam = self._camera()
        st = _lib.load().nsph_raycast_particles(grid.id, x.data_ptr(), radius.data_ptr(), n, ctypes.byref(cam),
                                                float(search_radius), float(step), int(max_steps),
                                                self._depth_buffer.data_ptr(), _lib.stream_handle(self.device))
        _lib.check(st, "SensorRaycast.update")

    def _clamp_no_hits(self) -> None:
        st = _lib.load().nsph_raycast_clamp_no_hits(self._depth_buffer.data_ptr(), self._depth_buffer.numel(),
                                                    float(self.max_distance), _lib.stream_handle(self.device))
        _lib.check(st, "SensorRaycast.update")

    def get_depth_image(self) -> torch.Tensor:
        """The depth image (height, width): > 0 the distance to the nearest
        surface, -1 no hit."""
        return self.depth_image

    def get_depth_image_numpy(self) -> np.ndarray:
        return self.depth_image.cpu().numpy()

    def update_camera_pose(self, position=None, direction=None, up=None) -> None:
        if position is not None:
            self.camera_position = np.array(position, dtype=np.float32)
        if direction is not None or up is not None:
            d = np.array(direction, dtype=np.float32) if direction is not None else self.camera_direction
            u = np.array(up, dtype=np.float32) if up is not None else self.camera_up
            self._compute_camera_basis(d, u)

    def update_camera_parameters(self, fov_radians: float | None = None, width: int | None = None,
                                 height: int | None = None, max_distance: float | None = None) -> None:
        recreate = False
        if width is not None and width != self.width:
            self.width = int(width)
            recreate = True
        if height is not None and height != self.height:
            self.height = int(height)
            recreate = True
        if fov_radians is not None:
            self.fov_radians = fov_radians
            self.fov_scale = math.tan(fov_radians * 0.5)
        if max_distance is not None:
            self.max_distance = max_distance
        if recreate:
            self.aspect_ratio = float(self.width) / float(self.height)
            self._depth_buffer = torch.zeros((self.height, self.width), dtype=torch.float32, device=self.device)
            self.depth_image = self._depth_buffer

    def point_camera_at(self, target, position=None, up=None) -> None:
        if position is not None:
            self.camera_position = np.array(position, dtype=np.float32)
        if up is None:
            up = np.array([0.0, 0.0, 1.0], dtype=np.float32)
        direction = np.array(target, dtype=np.float32) - self.camera_position
        self.update_camera_pose(position=self.camera_position, direction=direction, up=up)


__all__ = ["MAX_PARTICLE_RAY_MARCH_STEPS", "SensorRaycast", "camera_basis", "march_steps"]
