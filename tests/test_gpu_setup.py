"""Set-up on the device (imex_setup_dem / _cell_fract / _regrid through the C
ABI) against the oracle, bit for bit, and their error handling."""
import numpy as np
import pytest

import oracle as O
import setup_cases as S
from imex_sflow2d_v2_b200 import grid_setup as G
from imex_sflow2d_v2_b200.solver import ImexError

pytestmark = pytest.mark.gpu


def _raster(z, xll, yll, cs, nodata=-9999.0):
    return G.Raster(z.shape[0], z.shape[1], xll, yll, cs, nodata, z)


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


@pytest.mark.parametrize("name,dem,grid", S.DEM_CASES, ids=[c[0] for c in S.DEM_CASES])
def test_dem_sampling(name, dem, grid):
    ncols, nrows, xll, yll, cs = dem
    nx, ny, x0, y0, csz = grid
    z = S.dem_raster(ncols, nrows, xll, yll, cs, seed=sum(map(ord, name)), n_nodata=3)
    B, N = G.init_grid_topography(_raster(z, xll, yll, cs), nx, ny, x0, y0, csz, check=False)
    Bo, No, st = O.setup_dem(z, xll, yll, cs, -9999.0, nx, ny, x0, y0, csz)
    assert st == 0
    assert _same(B, Bo)
    assert np.array_equal(N, No)


def test_dem_sampling_large():
    # a 1500 x 1300 DEM at 7 m onto a 2000 x 1700 grid at 5 m
    z = S.dem_raster(1500, 1300, 0.0, 0.0, 7.0, seed=11, n_nodata=50)
    t = {}
    B, N = G.init_grid_topography(_raster(z, 0.0, 0.0, 7.0), 2000, 1700, 4.0, 4.0, 5.0,
                                  check=False, timing=t)
    Bo, No, st = O.setup_dem(z, 0.0, 0.0, 7.0, -9999.0, 2000, 1700, 4.0, 4.0, 5.0)
    assert st == 0 and _same(B, Bo) and np.array_equal(N, No)
    assert N.sum() > 0 and t["kernel_ms"] > 0.0


def test_dem_errors():
    z = S.dem_raster(10, 10, 0.0, 0.0, 1.0, seed=1)
    with pytest.raises(ImexError):      # cell centres west of the first node
        G.init_grid_topography(_raster(z, 0.0, 0.0, 1.0), 5, 5, -3.0, 0.0, 1.0, check=False)
    with pytest.raises(ImexError):      # one-node DEM
        G.init_grid_topography(_raster(np.ones((1, 1), order="F"), 0.0, 0.0, 1.0), 2, 2, 0.5,
                               0.5, 0.1, check=False)
    with pytest.raises(ValueError):     # the reference's own domain check
        G.init_grid_topography(_raster(z, 0.0, 0.0, 1.0), 5, 5, 0.0, 0.0, 1.0)


@pytest.mark.parametrize("name,grid,src", S.FRACT_CASES, ids=[c[0] for c in S.FRACT_CASES])
def test_cell_fract(name, grid, src):
    out = G.compute_cell_fract(*grid, *src)
    assert _same(out, O.cell_fract(*grid, *src))


def test_cell_fract_collapse_large():
    # a collapse of 600 m radius on a 5 m grid: 240 x 240 candidate cells
    args = (512, 512, 0.0, 0.0, 5.0, 1300.0, 1250.0, 600.0, 600.0, 0.0)
    t = {}
    out = G.compute_cell_fract(*args, timing=t)
    assert _same(out, O.cell_fract(*args))
    assert t["kernel_ms"] > 0.0


@pytest.mark.parametrize("name,ras,grid", S.REGRID_CASES, ids=[c[0] for c in S.REGRID_CASES])
def test_regrid(name, ras, grid):
    ncols, nrows, xll, yll, cs = ras
    fin = S.restart_raster(ncols, nrows, seed=len(name))
    out = G.regrid_scalar(_raster(fin, xll, yll, cs), *grid)
    ref, st = O.regrid(fin, xll, yll, cs, -9999.0, *grid)
    assert st == 0 and _same(out, ref)


def test_regrid_large():
    fin = S.restart_raster(1200, 900, seed=5)
    out = G.regrid_scalar(_raster(fin, -3.0, 2.0, 2.5), 1000, 800, 0.0, 5.0, 3.0)
    ref, st = O.regrid(fin, -3.0, 2.0, 2.5, -9999.0, 1000, 800, 0.0, 5.0, 3.0)
    assert st == 0 and _same(out, ref)
