"""HashGrid parity on the GPU: build (cell ids, permutation, cell ranges)
and the Warp-order query, bit-exact against the CPU oracle's restatement of
wp.HashGrid (newton/_src/sim/builder.py:9853,
newton/_src/solvers/xpbd/solver_xpbd.py:139,315-319,
newton/_src/solvers/semi_implicit/kernels_contact.py:54,68,71)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _points(n, seed, lo=-0.1, hi=0.6, special=False):
    rng = np.random.default_rng(seed)
    pts = (rng.random((n, 3)) * (hi - lo) + lo).astype(np.float32)
    if special and n > 8:
        pts[0] = [np.nan, 0.1, 0.1]
        pts[1] = [np.inf, -np.inf, 0.2]
        pts[2] = [1e30, -1e30, 3e9]
        pts[3] = [0.0, -0.0, 0.05]
        pts[4] = pts[5]  # duplicate position
    return pts


def _grid_arrays(grid):
    return {k: getattr(grid, k).cpu().numpy() for k in ("point_cells", "point_ids", "cell_starts", "cell_ends")}


@pytest.mark.parametrize("dims", [(128, 128, 128), (7, 5, 6), (256, 128, 128), (1, 1, 1)])
@pytest.mark.parametrize("n", [0, 1, 2, 1000, 4097, 70001])
def test_build_matches_oracle(oracle_mod, dims, n):
    from newton_sph_dev_b200 import HashGrid

    pts = _points(n, seed=n + dims[0], special=True)
    radius = 0.037
    grid = HashGrid(*dims, device=DEV)
    grid.reserve(max(n, 1))
    grid.build(torch.from_numpy(pts).to(DEV), radius)
    torch.cuda.synchronize()
    got = _grid_arrays(grid)
    ref = oracle_mod.grid_build(pts, radius, dims)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_rebuild_clears_previous_ranges(oracle_mod):
    from newton_sph_dev_b200 import HashGrid

    dims = (32, 32, 32)
    grid = HashGrid(*dims, device=DEV)
    a = _points(20000, 1)
    b = _points(3000, 2, lo=0.2, hi=0.9)
    grid.build(torch.from_numpy(a).to(DEV), 0.05)
    grid.build(torch.from_numpy(b).to(DEV), 0.05)
    torch.cuda.synchronize()
    got = _grid_arrays(grid)
    ref = oracle_mod.grid_build(b, 0.05, dims)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # and an empty rebuild leaves every cell empty
    grid.build(torch.zeros((0, 3), dtype=torch.float32, device=DEV), 0.05)
    torch.cuda.synchronize()
    assert int(grid.cell_starts.abs().sum()) == 0 and int(grid.cell_ends.abs().sum()) == 0


def test_rebuilds_across_the_sort_tile_sizes(oracle_mod):
    """Builds of at most 262,144 points sort in 512-key tiles, larger ones in
    2048-key tiles; each rebuild clears the previous build's cells in its own
    tile size. Alternating sizes across that boundary (exactly at it, one
    above, far above and far below) gives the oracle's grid every time."""
    from newton_sph_dev_b200 import HashGrid

    dims = (128, 128, 128)
    radius = 0.02
    grid = HashGrid(*dims, device=DEV)
    grid.reserve(400000)
    for i, n in enumerate([262144, 262145, 400000, 5000, 300001, 262144, 1]):
        pts = _points(n, seed=100 + i, lo=-0.3 + 0.1 * i, hi=1.2 + 0.1 * i)
        grid.build(torch.from_numpy(pts).to(DEV), radius)
        torch.cuda.synchronize()
        got = _grid_arrays(grid)
        ref = oracle_mod.grid_build(pts, radius, dims)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"build {i} (n={n}): {k}")


@pytest.mark.parametrize("dims,radius,qradius", [((128, 128, 128), 0.05, 0.05), ((16, 8, 4), 0.05, 0.12),
                                                 ((64, 64, 64), 0.1, 0.03)])
def test_query_matches_oracle(oracle_mod, dims, radius, qradius):
    from newton_sph_dev_b200 import HashGrid

    pts = _points(5000, 7)
    q = _points(300, 8, lo=-0.2, hi=0.7)
    grid = HashGrid(*dims, device=DEV)
    grid.build(torch.from_numpy(pts).to(DEV), radius)
    offsets, ids = grid.query(torch.from_numpy(q).to(DEV), qradius)
    offsets, ids = offsets.cpu().numpy(), ids.cpu().numpy()
    ref = oracle_mod.grid_build(pts, radius, dims)
    inv = np.float32(1.0) / np.float32(radius)
    for t in range(len(q)):
        expect = oracle_mod.grid_query(ref, dims, inv, q[t], qradius)
        np.testing.assert_array_equal(ids[offsets[t]:offsets[t + 1]], expect, err_msg=f"query {t}")


def test_capacity_and_argument_errors():
    from newton_sph_dev_b200 import _lib

    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.nsph_grid_create(8, 8, 8, 0, ctypes.byref(h)) == 0
    try:
        assert L.nsph_grid_reserve(h, 10) == 0
        pts = torch.zeros((11, 3), dtype=torch.float32, device=DEV)
        assert L.nsph_grid_build(h, pts.data_ptr(), 11, 0.1, None) == _lib.NSPH_ERR_CAPACITY
        assert L.nsph_grid_build(h, pts.data_ptr(), 10, 0.0, None) == _lib.NSPH_ERR_INVALID_ARG
        assert L.nsph_grid_build(h, pts.data_ptr(), 10, float("nan"), None) == _lib.NSPH_ERR_INVALID_ARG
        assert b"radius" in L.nsph_last_error()
        q = torch.zeros((1, 3), dtype=torch.float32, device=DEV)
        cnt = torch.zeros(1, dtype=torch.int32, device=DEV)
        h2 = ctypes.c_void_p()
        assert L.nsph_grid_create(4, 4, 4, 0, ctypes.byref(h2)) == 0
        assert L.nsph_grid_query(h2, q.data_ptr(), 1, 0.1, cnt.data_ptr(), None, None, None) == _lib.NSPH_ERR_NOT_BUILT
        L.nsph_grid_destroy(h2)
        assert L.nsph_grid_create(0, 4, 4, 0, ctypes.byref(h2)) == _lib.NSPH_ERR_INVALID_ARG
    finally:
        L.nsph_grid_destroy(h)


def test_model_grid_is_128_cubed():
    from conftest import lattice_scene

    model, _ = lattice_scene((4, 4, 4), device=DEV)
    assert model.particle_grid is not None
    assert (model.particle_grid.dim_x, model.particle_grid.dim_y, model.particle_grid.dim_z) == (128, 128, 128)
    model.particle_grid.reserve(model.particle_count)
    model.particle_grid.build(model.particle_q, 0.2)
    ids = model.particle_grid.point_ids.cpu().numpy()
    assert sorted(ids.tolist()) == list(range(model.particle_count))


def test_counting_and_radix_builds_alternate(oracle_mod):
    """Single-world grids build by cell counts when the table holds at most 16
    cells per point, else by the radix sort. Builds that alternate between
    the two on one grid, and repeated counting builds (whose per-cell counts
    must return to zero), all match the oracle."""
    from newton_sph_dev_b200 import HashGrid

    dims = (64, 64, 64)  # 262,144 cells
    grid = HashGrid(*dims, device=DEV)
    for n, seed in ((20000, 1), (25000, 2), (10000, 3), (30000, 4), (5000, 5), (20000, 6)):
        pts = _points(n, seed)
        grid.build(torch.from_numpy(pts).to(DEV), 0.02)
        torch.cuda.synchronize()
        got = _grid_arrays(grid)
        ref = oracle_mod.grid_build(pts, 0.02, dims)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"n={n}: {k}")
        counting = dims[0] * dims[1] * dims[2] <= 16 * n
        launches = grid.last_launches() if callable(grid.last_launches) else grid.last_launches
        assert (launches == 5) == counting, (n, launches)


def test_counting_build_partial_tile(oracle_mod):
    """The counting build on a cell table whose size is not a multiple of the
    scan's 8192-cell tile (the last tile reads its counts one by one), over
    repeated builds (the per-cell and per-tile counts must return to zero):
    the same grid as the oracle's each time."""
    from newton_sph_dev_b200 import HashGrid

    dims = (61, 53, 47)  # 151,951 cells: 19 tiles, the last one partial
    grid = HashGrid(*dims, device=DEV)
    for n, seed in ((12000, 11), (20000, 12), (15000, 13), (150000, 14)):
        pts = _points(n, seed)
        grid.build(torch.from_numpy(pts).to(DEV), 0.02)
        torch.cuda.synchronize()
        assert grid.last_launches == 5
        got = _grid_arrays(grid)
        ref = oracle_mod.grid_build(pts, 0.02, dims)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"n={n}: {k}")
