"""ctypes binding of libnsph.so (the C ABI declared in include/nsph.h).

The library is the only compute path: there is no CPU fallback. Loading fails
loudly when the shared object is missing, and every entry point's status is
turned into a Python exception by :func:`check`.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

# NSPH_LIBRARY selects another build of the library (the bounds-checked
# libnsph_bounds.so, for instance); by default the in-tree libnsph.so
_LIB_PATH = Path(os.environ["NSPH_LIBRARY"]).resolve() if os.environ.get("NSPH_LIBRARY") else \
    Path(__file__).resolve().parent / "libnsph.so"

NSPH_OK = 0
NSPH_ERR_INVALID_ARG = 1
NSPH_ERR_CAPACITY = 2
NSPH_ERR_CUDA = 3
NSPH_ERR_NOT_BUILT = 4
NSPH_ERR_OUT_OF_MEMORY = 5

NSPH_STATUS_NONFINITE_INPUT = 1
NSPH_STATUS_NONFINITE_OUTPUT = 2
NSPH_STATUS_ZERO_DENSITY = 4
NSPH_STATUS_SURROGATE_TIMEOUT = 8

c_int_p = ctypes.POINTER(ctypes.c_int)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_void_p = ctypes.c_void_p


class NsphGridView(ctypes.Structure):
    _fields_ = [
        ("point_cells", c_void_p),
        ("point_ids", c_void_p),
        ("cell_starts", c_void_p),
        ("cell_ends", c_void_p),
        ("cell_stride", ctypes.c_int),
        ("num_points", ctypes.c_int),
        ("dim_x", ctypes.c_int),
        ("dim_y", ctypes.c_int),
        ("dim_z", ctypes.c_int),
        ("cell_width", ctypes.c_float),
        ("cell_width_inv", ctypes.c_float),
        ("built", ctypes.c_int),
    ]


class NsphSphParams(ctypes.Structure):
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


class NsphContactParams(ctypes.Structure):
    """Layout of nsph_contact_params (include/nsph.h)."""

    _fields_ = [
        ("k_contact", ctypes.c_float),
        ("k_damp", ctypes.c_float),
        ("k_friction", ctypes.c_float),
        ("k_mu", ctypes.c_float),
        ("k_cohesion", ctypes.c_float),
        ("max_radius", ctypes.c_float),
    ]


class NsphShape(ctypes.Structure):
    """Layout of nsph_shape (include/nsph.h): one static analytic shape."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("flags", ctypes.c_int),
        ("world", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("pos", ctypes.c_float * 3),
        ("rot", ctypes.c_float * 4),
        ("scale", ctypes.c_float * 3),
        ("ke", ctypes.c_float),
        ("kd", ctypes.c_float),
        ("kf", ctypes.c_float),
        ("mu", ctypes.c_float),
    ]


class NsphSoftContacts(ctypes.Structure):
    """Layout of nsph_soft_contacts (include/nsph.h): device array pointers."""

    _fields_ = [
        ("count", c_void_p),
        ("particle", c_void_p),
        ("shape", c_void_p),
        ("body_pos", c_void_p),
        ("body_vel", c_void_p),
        ("normal", c_void_p),
        ("max", ctypes.c_int),
    ]


class NsphSoftContactParams(ctypes.Structure):
    """Layout of nsph_soft_contact_params (include/nsph.h)."""

    _fields_ = [
        ("ke", ctypes.c_float),
        ("kd", ctypes.c_float),
        ("kf", ctypes.c_float),
        ("mu", ctypes.c_float),
        ("adhesion", ctypes.c_float),
        ("restitution", ctypes.c_float),
        ("relaxation", ctypes.c_float),
        ("dt", ctypes.c_float),
    ]


class NsphRaycastCamera(ctypes.Structure):
    """Layout of nsph_raycast_camera (include/nsph.h)."""

    _fields_ = [
        ("position", ctypes.c_float * 3),
        ("direction", ctypes.c_float * 3),
        ("up", ctypes.c_float * 3),
        ("right", ctypes.c_float * 3),
        ("fov_scale", ctypes.c_float),
        ("aspect_ratio", ctypes.c_float),
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
        ("max_distance", ctypes.c_float),
    ]


# (name, restype, argtypes) of every exported entry point, in header order.
SIGNATURES = [
    ("nsph_version", ctypes.c_int, []),
    ("nsph_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("nsph_last_error", ctypes.c_char_p, []),
    ("nsph_build_flags", ctypes.c_int, []),
    ("nsph_debug_bounds_violations", ctypes.c_int, [ctypes.POINTER(ctypes.c_ulonglong)]),
    ("nsph_grid_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(c_void_p)]),
    ("nsph_grid_destroy", ctypes.c_int, [c_void_p]),
    ("nsph_grid_reserve", ctypes.c_int, [c_void_p, ctypes.c_int]),
    ("nsph_grid_build", ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_float, c_void_p]),
    ("nsph_grid_get_view", ctypes.c_int, [c_void_p, ctypes.POINTER(NsphGridView)]),
    ("nsph_grid_last_launches", ctypes.c_int, [c_void_p]),
    ("nsph_grid_query", ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, ctypes.c_float, c_void_p, c_void_p, c_void_p, c_void_p]),
    (
        "nsph_grid_build_noalloc",
        ctypes.c_int,
        [c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [c_void_p] * 5,
    ),
    (
        "nsph_integrate_particles",
        ctypes.c_int,
        [c_void_p] * 7 + [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, c_void_p, c_void_p, c_void_p],
    ),
    ("nsph_sph_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int * 3), ctypes.POINTER(c_void_p)]),
    ("nsph_sph_destroy", ctypes.c_int, [c_void_p]),
    (
        "nsph_sph_step",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 5
        + [c_void_p],
    ),
    (
        "nsph_sph_create_worlds",
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_void_p, ctypes.POINTER(c_void_p)],
    ),
    ("nsph_sph_set_world_params", ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int]),
    (
        "nsph_sph_step_worlds",
        ctypes.c_int,
        [c_void_p, ctypes.c_float, ctypes.c_int] + [c_void_p] * 8 + [ctypes.c_int] + [c_void_p] * 5 + [c_void_p],
    ),
    ("nsph_sph_enable_adjoint", ctypes.c_int, [c_void_p]),
    (
        "nsph_sph_step_adjoint",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 7
        + [c_void_p],
    ),
    (
        "nsph_sph_rollout",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int, ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 2
        + [c_void_p],
    ),
    (
        "nsph_sph_rollout_adjoint",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int, ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 4
        + [c_void_p],
    ),
    ("nsph_sph_reserve_segment", ctypes.c_int, [c_void_p, ctypes.c_int]),
    (
        "nsph_sph_segment_adjoint",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int, ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 4
        + [c_void_p],
    ),
    (
        "nsph_raycast_particles",
        ctypes.c_int,
        [c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.POINTER(NsphRaycastCamera), ctypes.c_float,
         ctypes.c_float, ctypes.c_int, c_void_p, c_void_p],
    ),
    ("nsph_raycast_clamp_no_hits", ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_float, c_void_p]),
    (
        "nsph_particle_contact_forces",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphContactParams), ctypes.c_int] + [c_void_p] * 5 + [c_void_p],
    ),
    (
        "nsph_particle_contact_deltas",
        ctypes.c_int,
        [c_void_p, ctypes.c_int] + [c_void_p] * 5 + [ctypes.c_float] * 5 + [c_void_p, c_void_p],
    ),
    (
        "nsph_fp32_peak",
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
         ctypes.POINTER(ctypes.c_float), c_void_p],
    ),
    ("nsph_soft_contacts_scratch_ints", ctypes.c_int, [ctypes.c_int]),
    (
        "nsph_soft_contacts_create",
        ctypes.c_int,
        [c_void_p, ctypes.c_int, ctypes.c_int] + [c_void_p] * 4
        + [ctypes.c_float, ctypes.POINTER(NsphSoftContacts), c_void_p, c_void_p],
    ),
    (
        "nsph_particle_shape_contact_forces",
        ctypes.c_int,
        [c_void_p, ctypes.c_int, ctypes.POINTER(NsphSoftContacts), ctypes.POINTER(NsphSoftContactParams)]
        + [c_void_p] * 5 + [c_void_p],
    ),
    (
        "nsph_particle_shape_contact_deltas",
        ctypes.c_int,
        [c_void_p, ctypes.c_int, ctypes.POINTER(NsphSoftContacts), ctypes.POINTER(NsphSoftContactParams)]
        + [c_void_p] * 6 + [c_void_p],
    ),
    (
        "nsph_particle_shape_restitution",
        ctypes.c_int,
        [ctypes.POINTER(NsphSoftContacts), ctypes.POINTER(NsphSoftContactParams)] + [c_void_p] * 6 + [c_void_p],
    ),
    (
        "nsph_apply_particle_deltas",
        ctypes.c_int,
        [ctypes.c_int] + [c_void_p] * 4 + [ctypes.c_float, ctypes.c_float, c_void_p, c_void_p, c_void_p],
    ),
    ("nsph_sph_enable_surrogate", ctypes.c_int, [c_void_p]),
    (
        "nsph_sph_features",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), ctypes.c_int]
        + [c_void_p] * 7
        + [ctypes.c_int]
        + [c_void_p] * 3
        + [c_void_p],
    ),
    ("nsph_sph_set_surrogate_launch", ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int]),
    ("nsph_sph_set_surrogate_wait_limit", ctypes.c_int, [c_void_p, ctypes.c_int]),
    (
        "nsph_sph_step_surrogate",
        ctypes.c_int,
        [c_void_p, ctypes.POINTER(NsphSphParams), c_void_p, ctypes.c_float, ctypes.c_int]
        + [c_void_p] * 8
        + [ctypes.c_int]
        + [c_void_p] * 5
        + [c_void_p],
    ),
    ("nsph_mlp_model_floats", ctypes.c_int, []),
    ("nsph_mlp_forward", ctypes.c_int, [ctypes.c_int, c_void_p, c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    ("nsph_mlp_gradient_ctas", ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    (
        "nsph_mlp_gradient",
        ctypes.c_int,
        [ctypes.c_int] + [c_void_p] * 4 + [ctypes.c_int, c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p],
    ),
    (
        "nsph_mlp_adam",
        ctypes.c_int,
        [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p] + [ctypes.c_float] * 4 + [ctypes.c_int, c_void_p],
    ),
    ("nsph_sph_neighbors", ctypes.c_int, [c_void_p, ctypes.POINTER(NsphSphParams), c_void_p, c_void_p, c_void_p, c_void_p]),
    ("nsph_sph_get_grid_view", ctypes.c_int, [c_void_p, ctypes.POINTER(NsphGridView)]),
    ("nsph_sph_enable_phase_timing", ctypes.c_int, [c_void_p, ctypes.c_int]),
    ("nsph_sph_phase_times", ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_float * 3)]),
    ("nsph_sph_adjoint_phase_times", ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_float * 5)]),
    ("nsph_sph_surrogate_phase_times", ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_float * 4)]),
    ("nsph_sph_set_launch", ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int]),
    ("nsph_sph_set_arithmetic", ctypes.c_int, [c_void_p, ctypes.c_int]),
    ("nsph_sph_last_launches", ctypes.c_int, [c_void_p]),
    ("nsph_sph_status", ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint), c_void_p]),
    ("nsph_sph_reset_status", ctypes.c_int, [c_void_p, c_void_p]),
]

_lib: ctypes.CDLL | None = None


class NsphError(RuntimeError):
    """A libnsph entry point returned a non-zero status."""

    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where} failed with status {status}: {message}")


def lib_path() -> Path:
    return _LIB_PATH


def load() -> ctypes.CDLL:
    """Load libnsph.so (once) and declare the C signatures.

    Raises:
        RuntimeError: the library has not been built (``__graft_entry__.build()``
            or ``python -m newton_sph_dev_b200._build``).
    """
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(
            f"{_LIB_PATH} is missing: build the CUDA library first "
            "(python -m newton_sph_dev_b200._build). There is no CPU fallback."
        )
    # the torch runtime must own the primary context before our statically
    # linked runtime touches it; importing torch first guarantees that order
    import torch  # noqa: F401

    lib = ctypes.CDLL(os.fspath(_LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().nsph_last_error()
    return msg.decode() if msg else ""


def check(status: int, where: str) -> None:
    """Raise the Newton-style exception for a non-zero status."""
    if status == NSPH_OK:
        return
    msg = last_error()
    if status in (NSPH_ERR_INVALID_ARG, NSPH_ERR_CAPACITY):
        raise ValueError(f"{where}: {msg}")
    raise NsphError(status, where, msg)


def ptr(t) -> int | None:
    """Raw device pointer of a tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(device) -> int:
    import torch

    return torch.cuda.current_stream(device).cuda_stream


NSPH_BUILD_BOUNDS_CHECK = 1


def bounds_checked() -> bool:
    """True when the loaded library is the bounds-checked build."""
    return bool(load().nsph_build_flags() & NSPH_BUILD_BOUNDS_CHECK)


def bounds_violations() -> int:
    """Index violations the bounds-checked build counted on the current
    device since the last call (0 in the release build)."""
    v = ctypes.c_ulonglong(0)
    check(load().nsph_debug_bounds_violations(ctypes.byref(v)), "bounds_violations")
    return int(v.value)
