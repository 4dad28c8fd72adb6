"""The allocation-free grid build, nsph_grid_build_noalloc.

Some callers cannot allocate device memory: code that rebuilds the grid
inside a CUDA stream capture, where cudaMalloc is not allowed, and programs
whose device memory belongs to another allocator. For them the library keeps
the sort scratch in a fixed device array and the caller passes every output.
This checks, through the C ABI, that two calls in a row give exactly what the
allocating path (HashGrid / nsph_grid_build) gives, and that sizes beyond the
fixed scratch are refused. The file is named to be collected last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _noalloc_build(lib, pts: torch.Tensor, radius: float, dims):
    n = int(pts.shape[0])
    nc = dims[0] * dims[1] * dims[2]
    cells = torch.full((max(n, 1),), -1, dtype=torch.int32, device=DEV)
    ids = torch.full((max(n, 1),), -1, dtype=torch.int32, device=DEV)
    starts = torch.full((nc,), 7, dtype=torch.int32, device=DEV)  # garbage the call must clear
    ends = torch.full((nc,), 7, dtype=torch.int32, device=DEV)
    st = lib.nsph_grid_build_noalloc(pts.data_ptr(), n, float(radius), *dims, cells.data_ptr(), ids.data_ptr(),
                                     starts.data_ptr(), ends.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return st, cells[:n], ids[:n], starts, ends


def _allocating_build(pts: torch.Tensor, radius: float, dims):
    from newton_sph_dev_b200 import HashGrid

    grid = HashGrid(*dims, device=DEV)
    grid.build(pts, radius)
    return grid.point_cells.clone(), grid.point_ids.clone(), grid.cell_starts.clone(), grid.cell_ends.clone()


def test_noalloc_build_matches_allocating_build_twice():
    from newton_sph_dev_b200 import _lib

    lib = _lib.load()
    dims = (64, 32, 48)
    rng = np.random.default_rng(123)
    # two calls in a row on different inputs: the second must not see the first's leftovers
    cases = [
        (torch.from_numpy((rng.random((100_000, 3)) * 1.2 - 0.1).astype(np.float32)).to(DEV), 0.03),
        (torch.from_numpy((rng.random((5_000, 3)) * 0.5).astype(np.float32)).to(DEV), 0.05),
    ]
    for pts, radius in cases:
        st, cells, ids, starts, ends = _noalloc_build(lib, pts, radius, dims)
        assert st == 0, _lib.last_error()
        ref = _allocating_build(pts, radius, dims)
        torch.cuda.synchronize()
        for got, want, name in zip((cells, ids, starts, ends), ref, ("point_cells", "point_ids", "cell_starts",
                                                                      "cell_ends")):
            assert torch.equal(got.cpu(), want.cpu()), name


def test_noalloc_build_refuses_more_points_than_its_scratch():
    from newton_sph_dev_b200 import _lib

    lib = _lib.load()
    limit = 1 << 18
    pts = torch.zeros((limit + 1, 3), dtype=torch.float32, device=DEV)
    st, *_ = _noalloc_build(lib, pts, 0.1, (8, 8, 8))
    assert st == _lib.NSPH_ERR_CAPACITY
    assert "NSPH_NOALLOC_MAX_POINTS" in _lib.last_error()


def test_noalloc_build_inside_a_graph_capture():
    """The reason the entry point exists: a build captured into a CUDA graph
    (no allocation, no synchronisation during the capture), replayed on new
    points copied into the captured input buffer."""
    from newton_sph_dev_b200 import _lib

    lib = _lib.load()
    dims = (32, 32, 32)
    radius = 0.04
    n = 20_000
    rng = np.random.default_rng(7)
    pts = torch.zeros((n, 3), dtype=torch.float32, device=DEV)
    cells = torch.zeros(n, dtype=torch.int32, device=DEV)
    ids = torch.zeros(n, dtype=torch.int32, device=DEV)
    starts = torch.zeros(dims[0] * dims[1] * dims[2], dtype=torch.int32, device=DEV)
    ends = torch.zeros_like(starts)
    # the warm-up call may be empty: it sets the device up all the same
    st = lib.nsph_grid_build_noalloc(pts.data_ptr(), 0, radius, *dims, cells.data_ptr(), ids.data_ptr(),
                                     starts.data_ptr(), ends.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 0, _lib.last_error()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    status = []
    with torch.cuda.graph(graph):
        status.append(lib.nsph_grid_build_noalloc(pts.data_ptr(), n, radius, *dims, cells.data_ptr(), ids.data_ptr(),
                                                  starts.data_ptr(), ends.data_ptr(),
                                                  torch.cuda.current_stream().cuda_stream))
    assert status == [0], _lib.last_error()
    for _ in range(2):
        new = torch.from_numpy((rng.random((n, 3)) * 1.1 - 0.05).astype(np.float32)).to(DEV)
        pts.copy_(new)
        graph.replay()
        torch.cuda.synchronize()
        ref = _allocating_build(new, radius, dims)
        for got, want, name in zip((cells, ids, starts, ends), ref, ("point_cells", "point_ids", "cell_starts",
                                                                      "cell_ends")):
            assert torch.equal(got.cpu(), want.cpu()), name
    del graph
