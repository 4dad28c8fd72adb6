"""HashGrid: the drop-in for ``wp.HashGrid`` (external warp-lang), as used by
Newton at newton/_src/sim/builder.py:9853 (``HashGrid(128, 128, 128)``),
newton/_src/solvers/xpbd/solver_xpbd.py:139 (``reserve``) and :315-319
(``build(points, radius)``), and queried from kernels at
newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71.

Backed by libnsph.so (include/nsph.h, ``nsph_grid_*``). Build semantics:
cell width = radius; cell coordinate = int(p * (1/radius)) (truncation);
physical cell = (c + 2^20) mod dim per axis; stable sort by cell id;
``cell_starts`` / ``cell_ends`` give each cell's range in sorted order.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


class _DeviceArray:
    """Zero-copy torch view of library-owned device memory."""

    def __init__(self, ptr: int, n: int, device: torch.device):
        self.__cuda_array_interface__ = {
            "shape": (n,),
            "typestr": "<i4",
            "data": (ptr, False),
            "version": 3,
            "strides": None,
        }
        self._device = device


def _view_int(ptr: int | None, n: int, device: torch.device, stride: int = 1) -> torch.Tensor:
    """int32 view of n library-owned elements spaced `stride` apart."""
    if not ptr or n == 0:
        return torch.zeros(0, dtype=torch.int32, device=device)
    flat = torch.as_tensor(_DeviceArray(ptr, (n - 1) * stride + 1, device), device=device)
    return flat[::stride] if stride != 1 else flat


class HashGrid:
    """Uniform hashed grid of ``dim_x * dim_y * dim_z`` cells on a CUDA device."""

    def __init__(self, dim_x: int, dim_y: int, dim_z: int, device: str | torch.device | None = None):
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        device = torch.device(device)
        if device.type != "cuda":
            raise ValueError("HashGrid needs a CUDA device (there is no CPU fallback)")
        self.device = device
        self.dim_x, self.dim_y, self.dim_z = int(dim_x), int(dim_y), int(dim_z)
        self.reserved = 0
        self._lib = _lib.load()
        handle = ctypes.c_void_p()
        _lib.check(
            self._lib.nsph_grid_create(self.dim_x, self.dim_y, self.dim_z, device.index or 0, ctypes.byref(handle)),
            "HashGrid()",
        )
        self._handle = handle

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.nsph_grid_destroy(h)
            self._handle = None

    @property
    def id(self) -> int:
        """Opaque handle (the C ``nsph_grid*``), like ``wp.HashGrid.id``."""
        return int(self._handle.value)

    def reserve(self, num_points: int) -> None:
        """Size the point buffers for up to `num_points` (allocates)."""
        _lib.check(self._lib.nsph_grid_reserve(self._handle, int(num_points)), "HashGrid.reserve")
        self.reserved = max(self.reserved, int(num_points))

    def build(self, points: torch.Tensor, radius: float) -> None:
        """Rebuild over `points` ((N, 3) float32 CUDA tensor) with cell width
        `radius`. Reserves on demand when N exceeds the reservation (outside
        of a CUDA graph capture, as the reference does)."""
        if points.dtype != torch.float32 or points.dim() != 2 or points.shape[1] != 3:
            raise ValueError("points must be an (N, 3) float32 tensor")
        if not points.is_cuda or points.device != self.device:
            raise ValueError(f"points must live on {self.device}")
        points = points.contiguous()
        n = int(points.shape[0])
        if n > self.reserved:
            self.reserve(n)
        st = self._lib.nsph_grid_build(self._handle, points.data_ptr(), n, float(radius),
                                       _lib.stream_handle(self.device))
        _lib.check(st, "HashGrid.build")

    @property
    def last_launches(self) -> int:
        """Kernels launched by the last build."""
        return int(self._lib.nsph_grid_last_launches(self._handle))

    # ---- host-visible views for tests and consumers --------------------
    def _view(self) -> _lib.NsphGridView:
        v = _lib.NsphGridView()
        _lib.check(self._lib.nsph_grid_get_view(self._handle, ctypes.byref(v)), "HashGrid.view")
        return v

    @property
    def num_points(self) -> int:
        return self._view().num_points

    @property
    def point_ids(self) -> torch.Tensor:
        """Sorted position -> original point index (hash_grid_point_id)."""
        v = self._view()
        return _view_int(v.point_ids, v.num_points, self.device)

    @property
    def point_cells(self) -> torch.Tensor:
        """Cell id of each point in sorted order."""
        v = self._view()
        return _view_int(v.point_cells, v.num_points, self.device)

    @property
    def cell_starts(self) -> torch.Tensor:
        """First sorted position of each cell (0 for empty cells)."""
        v = self._view()
        return _view_int(v.cell_starts, self.dim_x * self.dim_y * self.dim_z, self.device, v.cell_stride)

    @property
    def cell_ends(self) -> torch.Tensor:
        """One past the last sorted position of each cell (0 for empty cells)."""
        v = self._view()
        return _view_int(v.cell_ends, self.dim_x * self.dim_y * self.dim_z, self.device, v.cell_stride)

    def query(self, points: torch.Tensor, radius: float) -> tuple[torch.Tensor, torch.Tensor]:
        """Candidates of hash_grid_query(points[q], radius) for every q, in
        Warp's iteration order (no distance test).

        Returns:
            (offsets, ids): ids[offsets[q]:offsets[q+1]] are query q's candidates.
        """
        points = points.contiguous()
        nq = int(points.shape[0])
        counts = torch.zeros(nq, dtype=torch.int32, device=self.device)
        stream = _lib.stream_handle(self.device)
        _lib.check(self._lib.nsph_grid_query(self._handle, points.data_ptr(), nq, float(radius), counts.data_ptr(),
                                             None, None, stream), "HashGrid.query")
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=self.device)
        offsets[1:] = torch.cumsum(counts.to(torch.int64), 0)
        total = int(offsets[-1].item())
        ids = torch.empty(max(total, 1), dtype=torch.int32, device=self.device)
        if nq:
            _lib.check(self._lib.nsph_grid_query(self._handle, points.data_ptr(), nq, float(radius), None,
                                                 offsets.data_ptr(), ids.data_ptr(), stream), "HashGrid.query")
        return offsets, ids[:total]


__all__ = ["HashGrid"]
