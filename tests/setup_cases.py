"""Seeded set-up inputs (DEM rasters, sources, restart rasters) shared by the
oracle and GPU set-up tests, and numpy restatements of the three routines
(vectorised, same IEEE operations in the same order) that pin the oracle."""
import numpy as np


def dem_raster(ncols, nrows, xll, yll, cs, seed, nodata=-9999.0, n_nodata=0, negative=True):
    rng = np.random.default_rng(seed)
    x = np.arange(ncols)[:, None]
    y = np.arange(nrows)[None, :]
    z = 500.0 + 3.0 * x - 2.0 * y + 40.0 * np.sin(0.07 * x) * np.cos(0.05 * y)
    z = z + rng.normal(0.0, 5.0, size=(ncols, nrows))
    if negative:
        z[rng.random((ncols, nrows)) < 0.05] *= -1.0
    z = np.asfortranarray(z)
    if n_nodata:
        idx = rng.choice(ncols * nrows, size=n_nodata, replace=False)
        z[np.unravel_index(idx, z.shape, order="F")] = nodata
    return z


# (name, DEM (ncols, nrows, xll, yll, cs), grid (nx, ny, x0, y0, cell_size))
DEM_CASES = [
    ("same-res", (40, 30, 0.0, 0.0, 10.0), (38, 28, 5.0, 5.0, 10.0)),
    ("finer-dem", (90, 70, -3.0, 2.0, 4.0), (30, 22, 0.0, 5.0, 11.0)),
    ("coarser-dem", (12, 9, 100.0, 200.0, 25.0), (50, 37, 113.0, 213.0, 5.0)),
    ("offset", (33, 41, 0.25, -0.75, 1.0), (29, 36, 0.8, 0.1, 1.0)),
    ("one-column", (1, 25, 0.0, 0.0, 2.0), (1, 20, 1.0, 1.0, 2.0)),
    ("one-row", (25, 1, 0.0, 0.0, 2.0), (20, 1, 1.0, 1.0, 2.0)),
    ("grid-one-column", (20, 20, 0.0, 0.0, 1.0), (1, 15, 0.6, 0.6, 1.0)),
]

# (name, grid (nx, ny, x0, y0, cell_size), source (xs, ys, rs, r2s, angle))
FRACT_CASES = [
    ("circle", (24, 20, 0.0, 0.0, 10.0), (117.0, 93.0, 41.0, 41.0, 0.0)),
    ("rotated-ellipse", (30, 26, -50.0, 20.0, 7.5), (60.0, 110.0, 55.0, 23.0, 37.0)),
    ("edge", (16, 16, 0.0, 0.0, 5.0), (2.0, 40.0, 18.0, 9.0, 120.0)),
    ("sub-cell", (10, 10, 0.0, 0.0, 10.0), (44.3, 57.9, 2.5, 1.5, 15.0)),
    ("outside", (8, 8, 0.0, 0.0, 1.0), (100.0, 100.0, 2.0, 2.0, 0.0)),
]

# (name, raster (ncols, nrows, xll, yll, cs), grid (nx, ny, x0, y0, cell_size))
REGRID_CASES = [
    ("same-res", (30, 20, 0.0, 0.0, 5.0), (30, 20, 0.0, 0.0, 5.0)),
    ("finer-raster", (64, 48, -2.0, 1.0, 1.5), (20, 15, 0.0, 3.0, 4.0)),
    ("coarser-raster", (10, 8, 3.0, -1.0, 9.0), (40, 30, 5.0, 0.0, 2.0)),
    ("partial-cover", (12, 12, 10.0, 10.0, 3.0), (20, 20, 0.0, 0.0, 3.0)),
]


def restart_raster(ncols, nrows, seed, nodata=-9999.0):
    rng = np.random.default_rng(seed)
    f = rng.random((ncols, nrows)) * 3.0
    f[rng.random((ncols, nrows)) < 0.3] = 0.0
    f[rng.random((ncols, nrows)) < 0.05] = nodata
    return np.asfortranarray(f)


# ------------------------------------------------------------------ numpy
def _comp(o, d, n):
    J = np.arange(1, n + 1, dtype=np.float64)
    return 0.5 * ((o + (J - 1.0) * d) + (o + J * d))


def np_setup_dem(z, xll, yll, cs, nodata, nx, ny, x0, y0, cell_size):
    ncols, nrows = z.shape
    dx = cell_size if nx > 1 else 1.0
    dy = cell_size if ny > 1 else 1.0
    x1 = xll + (np.arange(1, ncols + 1, dtype=np.float64) - 0.5) * cs
    y1 = yll + (np.arange(1, nrows + 1, dtype=np.float64) - 0.5) * cs
    x2 = _comp(x0, dx, nx)[:, None] * np.ones((1, ny))
    y2 = _comp(y0, dy, ny)[None, :] * np.ones((nx, 1))
    zc = np.where(z > 0.0, z, 0.0)
    if ncols > 1:
        ix = np.minimum(np.floor((x2 - x1[0]) / (x1[1] - x1[0])).astype(np.int64) + 1, ncols - 1)
        ax = (x1[ix] - x2) / (x1[ix] - x1[ix - 1])
    else:
        ix = np.ones((nx, ny), dtype=np.int64)
        ax = np.zeros((nx, ny))
    if nrows > 1:
        iy = np.minimum(np.floor((y2 - y1[0]) / (y1[1] - y1[0])).astype(np.int64) + 1, nrows - 1)
        ay = (y1[iy] - y2) / (y1[iy] - y1[iy - 1])
    else:
        iy = np.ones((nx, ny), dtype=np.int64)
        ay = np.zeros((nx, ny))
    assert ix.min() >= 1 and iy.min() >= 1

    def Z(a, i, k):
        return a[i - 1, k - 1]
    if ncols == 1:
        nod = (Z(z, ix, iy) == nodata) | (Z(z, ix, iy + 1) == nodata)
        f = ay * Z(zc, ix, iy) + (1.0 - ay) * Z(zc, ix, iy + 1)
    elif nrows == 1:
        nod = (Z(z, ix, iy) == nodata) | (Z(z, ix + 1, iy) == nodata)
        f = ax * Z(zc, ix, iy) + (1.0 - ax) * Z(zc, ix + 1, iy)
    else:
        nod = ((Z(z, ix, iy) == nodata) | (Z(z, ix, iy + 1) == nodata)
               | (Z(z, ix + 1, iy) == nodata) | (Z(z, ix + 1, iy + 1) == nodata))
        f = (ax * (ay * Z(zc, ix, iy) + (1.0 - ay) * Z(zc, ix, iy + 1))
             + (1.0 - ax) * (ay * Z(zc, ix + 1, iy) + (1.0 - ay) * Z(zc, ix + 1, iy + 1)))
    return f, nod.astype(np.int8)


def np_cell_fract(nx, ny, x0, y0, cell_size, xs, ys, rs, r2s, angle):
    import math
    n = 200
    dx = cell_size if nx > 1 else 1.0
    dy = cell_size if ny > 1 else 1.0
    ang = ((angle / 180.0) * math.atan(1.0)) * 4.0
    ca, sa = math.cos(ang), math.sin(ang)
    h = np.arange(1, n + 1, dtype=np.float64)
    sub = (2.0 * h - 1.0) / (2.0 * n)
    xsub = np.tile((sub - 0.5) * dx, n)          # x index varies fastest
    ysub = np.repeat((sub - 0.5) * dy, n)
    R = rs if rs > r2s else r2s
    out = np.zeros((nx, ny))
    for j in range(1, nx + 1):
        xa, xb = x0 + (j - 1) * dx, x0 + j * dx
        xc = 0.5 * (xa + xb)
        for k in range(1, ny + 1):
            ya, yb = y0 + (k - 1) * dy, y0 + k * dy
            yc = 0.5 * (ya + yb)
            if xb < xs - R or xa > xs + R or yb < ys - R or ya > ys + R:
                continue
            X = (xc + xsub) - xs
            Y = (yc + ysub) - ys
            u = X * ca + Y * sa
            v = -(X * sa) + Y * ca
            cnt = int(np.count_nonzero((u * u) / (rs * rs) + (v * v) / (r2s * r2s) <= 1.0))
            out[j - 1, k - 1] = float(np.float32(cnt) / np.float32(n * n))
    return out


def np_regrid(fin, xll, yll, cs, nodata, nx, ny, x0, y0, cell_size):
    import math
    ncols, nrows = fin.shape
    f = np.where(fin == nodata, 0.0, fin)
    xin = xll + np.arange(ncols + 1, dtype=np.float64) * cs
    yin = yll + np.arange(nrows + 1, dtype=np.float64) * cs
    dX, dY = xin[1] - xin[0], yin[1] - yin[0]
    out = np.zeros((nx, ny))
    for j in range(1, nx + 1):
        xl, xr = x0 + (j - 1) * cell_size, x0 + j * cell_size
        ix1 = max(1, math.ceil((xl - xin[0]) / dX))
        ix2 = min(ncols, math.ceil((xr - xin[0]) / dX) + 1)
        for k in range(1, ny + 1):
            yl, yr = y0 + (k - 1) * cell_size, y0 + k * cell_size
            iy1 = max(1, math.ceil((yl - yin[0]) / dY))
            iy2 = min(nrows + 1, math.ceil((yr - yin[0]) / dY) + 1)
            s = 0.0
            for ix in range(ix1, ix2):
                ax = (min(xr, xin[ix]) - max(xl, xin[ix - 1])) / (xr - xl)
                for iy in range(iy1, iy2):
                    ay = (min(yr, yin[iy]) - max(yl, yin[iy - 1])) / (yr - yl)
                    s = s + ax * ay * f[ix - 1, iy - 1]
            out[j - 1, k - 1] = s
    return out
