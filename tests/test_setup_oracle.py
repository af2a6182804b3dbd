"""The oracle's set-up restatements (DEM sampling, compute_cell_fract,
restart regridding) against independent numpy restatements, bit for bit,
plus the analytic properties the reference itself prints or relies on."""
import math
import os

import numpy as np
import pytest

import oracle as O
import setup_cases as S


@pytest.mark.parametrize("name,dem,grid", S.DEM_CASES, ids=[c[0] for c in S.DEM_CASES])
def test_dem_sampling_matches_numpy(name, dem, grid):
    ncols, nrows, xll, yll, cs = dem
    nx, ny, x0, y0, csz = grid
    z = S.dem_raster(ncols, nrows, xll, yll, cs, seed=sum(map(ord, name)), n_nodata=3)
    B, N, st = O.setup_dem(z, xll, yll, cs, -9999.0, nx, ny, x0, y0, csz)
    assert st == 0
    Bn, Nn = S.np_setup_dem(z, xll, yll, cs, -9999.0, nx, ny, x0, y0, csz)
    assert np.array_equal(B.view(np.int64), Bn.view(np.int64))
    assert np.array_equal(N, Nn)
    if min(ncols, nrows, nx, ny) > 1:
        assert N.sum() > 0       # the planted NODATA nodes reach the grid


def test_dem_sampling_reproduces_a_plane():
    # bilinear interpolation is exact for a plane (heights kept positive)
    ncols, nrows, cs = 50, 40, 2.0
    xc = (np.arange(1, ncols + 1) - 0.5) * cs
    yc = (np.arange(1, nrows + 1) - 0.5) * cs
    z = np.asfortranarray(100.0 + 0.5 * xc[:, None] - 0.25 * yc[None, :])
    B, N, st = O.setup_dem(z, 0.0, 0.0, cs, -9999.0, 40, 30, 3.0, 3.0, 2.0)
    assert st == 0 and not N.any()
    x = 3.0 + (np.arange(40) + 0.5) * 2.0
    y = 3.0 + (np.arange(30) + 0.5) * 2.0
    np.testing.assert_allclose(B, 100.0 + 0.5 * x[:, None] - 0.25 * y[None, :], rtol=0, atol=1e-11)


def test_dem_outside_is_flagged():
    z = S.dem_raster(10, 10, 0.0, 0.0, 1.0, seed=1)
    _, _, st = O.setup_dem(z, 0.0, 0.0, 1.0, -9999.0, 5, 5, -3.0, 0.0, 1.0)
    assert st & 1


@pytest.mark.parametrize("name,grid,src", S.FRACT_CASES, ids=[c[0] for c in S.FRACT_CASES])
def test_cell_fract_matches_numpy(name, grid, src):
    out = O.cell_fract(*grid, *src)
    ref = S.np_cell_fract(*grid, *src)
    assert np.array_equal(out.view(np.int64), ref.view(np.int64))
    assert out.min() >= 0.0 and out.max() <= 1.0


def test_cell_fract_area():
    # the reference's own check: dx*dy*SUM(cell_fract) against pi*rs*r2s
    nx, ny, x0, y0, cs = 40, 40, 0.0, 0.0, 5.0
    rs, r2s = 60.0, 35.0
    out = O.cell_fract(nx, ny, x0, y0, cs, 100.0, 100.0, rs, r2s, 25.0)
    area = cs * cs * out.sum()
    assert abs(1.0 - area / (math.pi * rs * r2s)) < 1e-3
    # cells fully inside count 40000/40000
    assert (out == 1.0).sum() > 100


@pytest.mark.parametrize("name,ras,grid", S.REGRID_CASES, ids=[c[0] for c in S.REGRID_CASES])
def test_regrid_matches_numpy(name, ras, grid):
    ncols, nrows, xll, yll, cs = ras
    fin = S.restart_raster(ncols, nrows, seed=len(name))
    out, st = O.regrid(fin, xll, yll, cs, -9999.0, *grid)
    assert st == 0
    ref = S.np_regrid(fin, xll, yll, cs, -9999.0, *grid)
    assert np.array_equal(out.view(np.int64), ref.view(np.int64))


def test_regrid_same_grid_is_identity_but_last_column():
    # with the raster on the grid itself every cell takes its own value,
    # except the last column: the reference's ix2 <= ncols never reads it
    fin = S.restart_raster(12, 9, seed=3, nodata=-1.0e30)
    out, st = O.regrid(fin, 0.0, 0.0, 2.0, -1.0e30, 12, 9, 0.0, 0.0, 2.0)
    assert st == 0
    want = np.where(fin == -1.0e30, 0.0, fin)
    np.testing.assert_allclose(out[:-1], want[:-1], rtol=1e-15, atol=0)
    assert not out[-1].any()


def test_esri_round_trip(tmp_path):
    from imex_sflow2d_v2_b200.grid_setup import Raster, read_esri_ascii, write_esri_ascii
    z = np.asfortranarray(np.arange(12, dtype=np.float64).reshape(4, 3, order="F"))
    r = Raster(4, 3, 10.0, 20.0, 5.0, -9999.0, z)
    p = os.path.join(tmp_path, "d.asc")
    write_esri_ascii(p, r, fmt="%.17g")
    rr = read_esri_ascii(p)
    assert (rr.ncols, rr.nrows, rr.xllcorner, rr.yllcorner, rr.cellsize) == (4, 3, 10.0, 20.0, 5.0)
    assert np.array_equal(rr.z, z)
    # the first line written is the northernmost row (k = nrows)
    with open(p) as f:
        lines = f.read().splitlines()
    assert lines[6].split() == ["8", "9", "10", "11"]
