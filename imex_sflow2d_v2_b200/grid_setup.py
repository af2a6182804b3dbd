"""Set-up on the device: DEM sampling, source/collapse cell fractions and
restart regridding, through the C ABI (imex_setup_*).

Mirrors the reference's set-up routines:
- ``read_esri_ascii``: the DEM/restart reader's header and row order
  (src/inpout_2d.f90:3516-3605, 5140-5190);
- ``init_grid_topography``: init_grid's B_nodata / B_cent sampling with its
  domain checks (src/inpout_2d.f90:3523-3563, src/geometry_2d.f90:320-342);
- ``compute_cell_fract`` (src/geometry_2d.f90:1678-1773);
- ``regrid_scalar`` over a whole grid, as read_solution applies it to a
  restart raster (src/inpout_2d.f90:5203-5246).

Arrays use the reference's column-major layouts: (ncols, nrows) rasters
with row 1 the southernmost, (nx, ny) grids.  The work runs on the GPU;
there is no CPU path (the library raises if it cannot run).
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from .abi import IMEX_OK
from .solver import ImexError, load_library


@dataclass
class Raster:
    """An ESRI ASCII grid: z[j, k] for column j (west to east) and row k
    (south to north), both 0-based here."""
    ncols: int
    nrows: int
    xllcorner: float
    yllcorner: float
    cellsize: float
    nodata: float
    z: np.ndarray


def read_esri_ascii(path):
    """Six header lines (key value: ncols, nrows, xllcorner, yllcorner,
    cellsize, NODATA_value), then nrows lines from north to south; stored
    with row 1 the southernmost as the reference does
    (topography_profile(3,:,nrows-k+1) = line k)."""
    with open(path) as f:
        hdr = [f.readline().split() for _ in range(6)]
        vals = np.array(f.read().split(), dtype=np.float64)
    ncols, nrows = int(hdr[0][1]), int(hdr[1][1])
    xll, yll, cs, nd = (float(hdr[i][1]) for i in range(2, 6))
    if vals.size < ncols * nrows:
        raise ValueError("%s: %d values for a %dx%d grid" % (path, vals.size, ncols, nrows))
    rows = vals[:ncols * nrows].reshape(nrows, ncols)       # north first
    z = np.asfortranarray(rows[::-1].T)                      # (ncols, nrows), south first
    return Raster(ncols, nrows, xll, yll, cs, nd, z)


def write_esri_ascii(path, r, fmt="%.6g"):
    """Inverse of read_esri_ascii (rows written north first)."""
    with open(path, "w") as f:
        f.write("ncols %d\nnrows %d\nxllcorner %r\nyllcorner %r\ncellsize %r\nNODATA_value %r\n"
                % (r.ncols, r.nrows, r.xllcorner, r.yllcorner, r.cellsize, r.nodata))
        for k in range(r.nrows - 1, -1, -1):
            f.write(" ".join(fmt % v for v in r.z[:, k]) + "\n")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc, where):
    if rc != IMEX_OK:
        L = load_library()
        raise ImexError(rc, where, L.imex_setup_last_error().decode())


def check_domain(dem, nx, ny, x0, y0, cell_size):
    """The reference's DEM/domain checks (src/inpout_2d.f90:3523-3563); each
    failing one stops the reference, here it raises ValueError.  The last
    test is the reference's as written (it compares with yllcorner + 0.5 +
    nrows*cellsize and stops when the two are within 1e-10)."""
    xll, yll, cs = dem.xllcorner, dem.yllcorner, dem.cellsize
    if x0 - (xll + 0.5 * cs) < -1.0e-10:
        raise ValueError("Computational domain problem: x0 < xllcorner+0.5*cellsize")
    if x0 + nx * cell_size > xll + (0.5 + dem.ncols) * cs:
        raise ValueError("Computational domain problem: right edge > xllcorner+ncols*cellsize")
    if y0 - (yll + 0.5 * cs) < -1.0e-10:
        raise ValueError("Computational domain problem: y0 < yllcorner+0.5*cellsize")
    if abs((y0 + ny * cell_size) - (yll + 0.5 + dem.nrows * cs)) < 1.0e-10:
        raise ValueError("Computational domain problem: top edge > yllcorner+nrows*cellsize")


def init_grid_topography(dem, nx, ny, x0, y0, cell_size, device=-1, check=True, timing=None):
    """(B_cent, B_nodata) at the cell centres of the nx*ny grid.  `timing`
    (a dict) receives the kernel's device time in ms under 'kernel_ms'."""
    if check:
        check_domain(dem, nx, ny, x0, y0, cell_size)
    L = load_library()
    z = np.asfortranarray(dem.z, dtype=np.float64)
    B = np.zeros((nx, ny), dtype=np.float64, order="F")
    N = np.zeros((nx, ny), dtype=np.int8, order="F")
    ms = C.c_float(0.0)
    rc = L.imex_setup_dem(int(device), dem.ncols, dem.nrows, dem.xllcorner, dem.yllcorner,
                          dem.cellsize, dem.nodata, _dp(z), nx, ny, float(x0), float(y0),
                          float(cell_size), _dp(B), N.ctypes.data_as(C.POINTER(C.c_int8)),
                          C.byref(ms))
    _check(rc, "imex_setup_dem")
    if timing is not None:
        timing["kernel_ms"] = ms.value
    return B, N


def compute_cell_fract(nx, ny, x0, y0, cell_size, xs, ys, rs, r2s, angle, device=-1,
                       timing=None):
    """Share of each cell inside the ellipse (centre xs, ys; semi-axes rs,
    r2s; rotation `angle` in degrees), as the reference's 200x200 subgrid
    count in single precision."""
    L = load_library()
    out = np.zeros((nx, ny), dtype=np.float64, order="F")
    ms = C.c_float(0.0)
    rc = L.imex_setup_cell_fract(int(device), nx, ny, float(x0), float(y0), float(cell_size),
                                 float(xs), float(ys), float(rs), float(r2s), float(angle),
                                 _dp(out), C.byref(ms))
    _check(rc, "imex_setup_cell_fract")
    if timing is not None:
        timing["kernel_ms"] = ms.value
    return out


def regrid_scalar(raster, nx, ny, x0, y0, cell_size, device=-1, timing=None):
    """Area-weighted average of the raster over every grid cell (values equal
    to NODATA count as 0), with the reference's loop bounds."""
    L = load_library()
    fin = np.asfortranarray(raster.z, dtype=np.float64)
    out = np.zeros((nx, ny), dtype=np.float64, order="F")
    ms = C.c_float(0.0)
    rc = L.imex_setup_regrid(int(device), raster.ncols, raster.nrows, raster.xllcorner,
                             raster.yllcorner, raster.cellsize, raster.nodata, _dp(fin), nx, ny,
                             float(x0), float(y0), float(cell_size), _dp(out), C.byref(ms))
    _check(rc, "imex_setup_regrid")
    if timing is not None:
        timing["kernel_ms"] = ms.value
    return out
