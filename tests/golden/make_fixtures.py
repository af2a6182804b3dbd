"""Builds tests/golden/test2d_inputs.npz from the reference's TESTS/TEST_2D
inputs (restart file INIT_2D_0000.q_2d and topography_dem.asc), and
tests/golden/bw_box_inputs.npz from TESTS/TEST_BW and TESTS/TEST_BOX (400 x 1
grids: restart files and DEMs), read as text.

The restart is read as read_solution does (src/inpout_2d.f90:5418-5442:
q(1:n_vars,j,k) in j-fastest order, q1 <= 0 zeroes the cell, negative solids
are zeroed); the DEM is bilinearly interpolated to the cell centres as
interp_2d_scalar does (src/geometry_2d.f90:1172-1228) after
topography_profile is built from the ESRI header (src/inpout_2d.f90:3572-3605).
Only this script reads the reference tree; the tests read the .npz.

Usage: python tests/golden/make_fixtures.py /path/to/reference
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_q2d(path, nx, ny, nv):
    vals = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if parts:
                vals.append([float(x) for x in parts])
    a = np.array(vals)
    assert a.shape == (nx * ny, 2 + nv), a.shape
    q = np.zeros((nv, nx, ny))
    for c in range(nx * ny):
        j, k = c % nx, c // nx
        q[:, j, k] = a[c, 2:]
        if q[0, j, k] <= 0.0:
            q[:, j, k] = 0.0
        for i in range(4, nv):
            if q[i, j, k] <= 0.0:
                q[i, j, k] = 0.0
    return q


def read_asc(path):
    hdr = {}
    rows = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0].lower() in ("ncols", "nrows", "xllcorner", "yllcorner", "cellsize",
                                    "nodata_value"):
                hdr[parts[0].lower()] = float(parts[1])
            else:
                rows.append([float(x) for x in parts])
    ncols, nrows = int(hdr["ncols"]), int(hdr["nrows"])
    z = np.array(rows).reshape(nrows, ncols)
    # topography_profile(3,:,nrows-k+1) = row k
    prof = np.zeros((ncols, nrows))
    for k in range(nrows):
        prof[:, nrows - k - 1] = z[k]
    xs = hdr["xllcorner"] + (np.arange(1, ncols + 1) - 0.5) * hdr["cellsize"]
    ys = hdr["yllcorner"] + (np.arange(1, nrows + 1) - 0.5) * hdr["cellsize"]
    return xs, ys, np.maximum(prof, 0.0)


def interp(xs, ys, f, x2, y2):
    """interp_2d_scalar, including its one-row and one-column branches."""
    if len(xs) > 1:
        ix = math.floor((x2 - xs[0]) / (xs[1] - xs[0])) + 1
        ix = min(ix, len(xs) - 1)
        ax = (xs[ix] - x2) / (xs[ix] - xs[ix - 1])
    else:
        ix, ax = 1, 0.0
    if len(ys) > 1:
        iy = math.floor((y2 - ys[0]) / (ys[1] - ys[0])) + 1
        iy = min(iy, len(ys) - 1)
        ay = (ys[iy] - y2) / (ys[iy] - ys[iy - 1])
    else:
        iy, ay = 1, 0.0
    if len(xs) == 1:
        return ay * f[ix - 1, iy - 1] + (1.0 - ay) * f[ix - 1, iy]
    if len(ys) == 1:
        return ax * f[ix - 1, iy - 1] + (1.0 - ax) * f[ix, iy - 1]
    return (ax * (ay * f[ix - 1, iy - 1] + (1.0 - ay) * f[ix - 1, iy])
            + (1.0 - ax) * (ay * f[ix, iy - 1] + (1.0 - ay) * f[ix, iy]))


def grid_b_cent(ref_dir, nx, ny, cs, x0, y0):
    """B_cent at the cell centres (a direction of one cell has spacing 1,
    src/geometry_2d.f90:250-266)."""
    xs, ys, prof = read_asc(os.path.join(ref_dir, "topography_dem.asc"))
    dx = cs if nx > 1 else 1.0
    dy = cs if ny > 1 else 1.0
    xst = x0 + np.arange(nx + 1) * dx
    yst = y0 + np.arange(ny + 1) * dy
    xc = 0.5 * (xst[:-1] + xst[1:])
    yc = 0.5 * (yst[:-1] + yst[1:])
    B = np.zeros((nx, ny))
    for k in range(ny):
        for j in range(nx):
            B[j, k] = interp(xs, ys, prof, xc[j], yc[k])
    return B


def main(ref):
    d = os.path.join(ref, "TESTS", "TEST_2D")
    nx, ny, nv, cs, x0, y0 = 100, 68, 5, 0.3, 0.0, -10.2
    q = read_q2d(os.path.join(d, "INIT_2D_0000.q_2d"), nx, ny, nv)
    xs, ys, prof = read_asc(os.path.join(d, "topography_dem.asc"))
    xst = x0 + np.arange(nx + 1) * cs
    yst = y0 + np.arange(ny + 1) * cs
    xc = 0.5 * (xst[:-1] + xst[1:])
    yc = 0.5 * (yst[:-1] + yst[1:])
    B = np.zeros((nx, ny))
    for k in range(ny):
        for j in range(nx):
            B[j, k] = interp(xs, ys, prof, xc[j], yc[k])
    np.savez_compressed(os.path.join(HERE, "test2d_inputs.npz"), q=q, B_cent=B,
                        nx=nx, ny=ny, cell_size=cs, x0=x0, y0=y0)
    print("wrote test2d_inputs.npz", q.shape, float(q[0].sum()), float(B.min()), float(B.max()))
    # TESTS/TEST_BW (inflow from the west) and TESTS/TEST_BOX (a released
    # box): 400 x 1 cells of 125 m, one solid class, restart files and DEMs
    out = {}
    for name, restart in (("bw", "INIT_BW_0000.q_2d"), ("box", "INIT_BOX_0000.q_2d")):
        d = os.path.join(ref, "TESTS", "TEST_" + name.upper())
        nx, ny, nv, cs, x0, y0 = 400, 1, 5, 125.0, 0.0, 0.0
        out[name + "_q"] = read_q2d(os.path.join(d, restart), nx, ny, nv)
        out[name + "_B_cent"] = grid_b_cent(d, nx, ny, cs, x0, y0)
    np.savez_compressed(os.path.join(HERE, "bw_box_inputs.npz"), nx=400, ny=1, cell_size=125.0,
                        x0=0.0, y0=0.0, **out)
    print("wrote bw_box_inputs.npz", {k: float(np.abs(v).sum()) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
