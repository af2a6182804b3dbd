"""Run set-up for the IMEX time step: parameters, static planes, initial state.

This module is the host-side set-up that the reference performs once before
its time loop (namelist defaults, grid, topography derivatives, inlet cells,
inlet state).  It is not on the time-step path: its outputs are the inputs of
the C ABI (include/imex_gpu.h).  Each function names the reference routine it
restates.  The benchmark workloads are built here from seeded synthetic data
(no dataset is involved).
"""
import math

import numpy as np

from .abi import IMEX_ABI_VERSION, IMEX_MAX_SOLID, ImexParams

EPSILON = np.finfo(np.float64).eps


def default_params(nx, ny, n_solid, cell_size, x0=0.0, y0=0.0):
    """Namelist defaults of init_param (src/inpout_2d.f90:393-525) plus the
    gas-transport values used by the reference test inputs."""
    p = ImexParams()
    p.abi_version = IMEX_ABI_VERSION
    p.nx, p.ny, p.n_solid = nx, ny, n_solid
    p.x0, p.y0, p.cell_size = x0, y0, cell_size
    dx = cell_size if nx > 1 else 1.0
    dy = cell_size if ny > 1 else 1.0
    # src/geometry_2d.f90:286-290
    p.eps_sing = min(min(dx ** 4.0, dy ** 4.0), 1.0e-10)
    p.n_rk = 2
    nv = 4 + n_solid
    for i in range(nv):
        p.limiter[i] = 1
    p.limiter[nv] = p.limiter[1]       # src/inpout_2d.f90:2079-2080
    p.limiter[nv + 1] = p.limiter[2]
    p.cfl = 0.24
    p.max_dt = 1.0e-3
    p.reconstr_coeff = 1.0
    p.theta = 1.0
    p.energy_flag = 1
    p.alpha_flag = 0
    p.gas_flag = 1
    p.liquid_flag = 0
    p.rheology_flag = 0
    p.rheology_model = 0
    p.grav = 9.81
    p.T_ambient = 300.0
    p.pres = 101300.0
    p.sp_heat_a = 998.0
    p.sp_gas_const_a = 287.051
    p.kin_visc_c = 1.48e-5
    p.maximum_solid_packing = 0.64
    p.mu = -1.0
    p.xi = -1.0
    p.friction_factor = 0.0
    for i in range(4):
        p.time_param[i] = 1.0e30
    p.time_param[2] = 0.0
    p.T_erodible = 300.0
    p.erodible_porosity = 0.0
    for i in range(n_solid):
        p.erodible_fract[i] = 1.0 / n_solid
    return p


def set_bc(p, side, var, flag, value=0.0):
    bc = getattr(p, "bc" + side)
    bc[var].flag = flag
    bc[var].value = value


def transmissive_bcs(p):
    """H: one-sided slope (flag 2); HU, HV, T: zero Neumann; alphas: one-sided
    slope -- the boundary set of TESTS/TEST_DAMBREAK/*/IMEX_SfloW2D.inp."""
    nv = 4 + p.n_solid
    for side in "WESN":
        set_bc(p, side, 0, 2)
        set_bc(p, side, 1, 1, 0.0)
        set_bc(p, side, 2, 1, 0.0)
        set_bc(p, side, 3, 1, 0.0)
        for i in range(4, nv):
            set_bc(p, side, i, 2)


def zero_gradient_bcs(p):
    """Every variable zero-gradient Neumann (flag 1, value 0) on every side --
    the boundary set of the reference's ensemble example
    (EXAMPLES/EXAMPLE_ENSEMBLE_ETNA/templatedir/IMEX_SfloW2D.inp:42-87)."""
    for side in "WESN":
        for i in range(4 + p.n_solid):
            set_bc(p, side, i, 1, 0.0)


def grid(p):
    """x_stag, x_comp, y_stag, y_comp as in init_grid (geometry_2d.f90:292-314)."""
    nx, ny = p.nx, p.ny
    dx = p.cell_size if nx > 1 else 1.0
    dy = p.cell_size if ny > 1 else 1.0
    x_stag = p.x0 + np.arange(nx + 1, dtype=np.float64) * dx
    y_stag = p.y0 + np.arange(ny + 1, dtype=np.float64) * dy
    x_comp = 0.5 * (x_stag[:-1] + x_stag[1:])
    y_comp = 0.5 * (y_stag[:-1] + y_stag[1:])
    return x_stag, x_comp, y_stag, y_comp


def topography_geom(B, dx, dy):
    """5-point first/second derivatives of topography_reconstruction
    (src/geometry_2d.f90:676-775); the 2-cell border copies the nearest
    interior value.  B is (nx, ny)."""
    nx, ny = B.shape
    c1 = [-2.0, -1.0, 0.0, 1.0, 2.0]
    c2 = [2.0, -1.0, -2.0, -1.0, 2.0]
    out = {}
    if (ny == 1 and nx >= 5) or (nx == 1 and ny >= 5):
        # a one-row (one-column) grid.  The reference's stencil loop runs over
        # rows 3..ny-2, none here, and its border copies then index rows 3,
        # 0 and -1 of the one-row arrays (src/geometry_2d.f90:700-790), so
        # its values are undefined; the planes below are the loop's stencil
        # applied along the row, with the cross-direction terms zero
        along_x = ny == 1
        b = B[:, 0] if along_x else B[0, :]
        n, d = len(b), (dx if along_x else dy)
        p1 = np.zeros(n)
        p2 = np.zeros(n)
        for kj in range(5):
            p1[2:n - 2] = p1[2:n - 2] + c1[kj] * b[kj:kj + n - 4]
            p2[2:n - 2] = p2[2:n - 2] + c2[kj] * b[kj:kj + n - 4]
        p1[2:n - 2] = p1[2:n - 2] / (10.0 * d)
        p2[2:n - 2] = p2[2:n - 2] / (7.0 * d ** 2)
        for a in (p1, p2):
            a[0] = a[1] = a[2]
            a[n - 1] = a[n - 2] = a[n - 3]
        shape = B.shape
        z = np.zeros(shape)
        first = np.asfortranarray(p1.reshape(shape))
        second = np.asfortranarray(p2.reshape(shape))
        out["B_prime_x_geom"] = first if along_x else z.copy()
        out["B_prime_y_geom"] = z.copy() if along_x else first
        out["B_second_xx_geom"] = second if along_x else z.copy()
        out["B_second_yy_geom"] = z.copy() if along_x else second
        out["B_second_xy_geom"] = z.copy()
        return out
    if nx < 5 or ny < 5:
        z = np.zeros((nx, ny))
        for n in ("B_prime_x_geom", "B_prime_y_geom", "B_second_xx_geom",
                  "B_second_xy_geom", "B_second_yy_geom"):
            out[n] = z.copy()
        return out
    J = slice(2, nx - 2)
    K = slice(2, ny - 2)
    bx = np.zeros((nx - 4, ny - 4))
    bxx = np.zeros_like(bx)
    by = np.zeros_like(bx)
    byy = np.zeros_like(bx)
    for kj in range(5):
        sh = B[kj:kj + nx - 4, 2:ny - 2]
        bx = bx + c1[kj] * sh
        bxx = bxx + c2[kj] * sh
    for kk in range(5):
        sh = B[2:nx - 2, kk:kk + ny - 4]
        by = by + c1[kk] * sh
        byy = byy + c2[kk] * sh
    bx = bx / (10.0 * dx)
    by = by / (10.0 * dy)
    bxx = bxx / (7.0 * dx ** 2)
    byy = byy / (7.0 * dy ** 2)
    # the 25-point mixed stencil is the outer product of c1 with itself; it is
    # applied as two 5-point passes (the sum order differs from the double
    # loop of the reference only in the last bits)
    tx = np.zeros((nx - 4, ny))
    for kj in range(5):
        tx = tx + c1[kj] * B[kj:kj + nx - 4, :]
    ws = np.zeros_like(bx)
    for kk in range(5):
        ws = ws + c1[kk] * tx[:, kk:kk + ny - 4]
    bxy = ws / ((10.0 * dx) * (10.0 * dy))
    jj = np.clip(np.arange(nx), 2, nx - 3) - 2
    kk_ = np.clip(np.arange(ny), 2, ny - 3) - 2
    for n, a in (("B_prime_x_geom", bx), ("B_prime_y_geom", by),
                 ("B_second_xx_geom", bxx), ("B_second_xy_geom", bxy),
                 ("B_second_yy_geom", byy)):
        out[n] = np.asfortranarray(a[np.ix_(jj, kk_)])
    del J, K
    return out


def slope_correction_planes(geom):
    """grav_coeff, d_grav_coeff_dx and the staggered grav_coeff from the
    *_geom derivatives (src/geometry_2d.f90:827-847)."""
    bx, by = geom["B_prime_x_geom"], geom["B_prime_y_geom"]
    bxx, bxy = geom["B_second_xx_geom"], geom["B_second_xy_geom"]
    gc = 1.0 / (1.0 + bx * bx + by * by)
    dgc = -(2.0 * (gc * gc) * (bx * bxx + by * bxy))
    nx, ny = gc.shape
    sx = np.empty((nx + 1, ny))
    sx[0] = gc[0]
    sx[1:nx] = 0.5 * (gc[:-1] + gc[1:])
    sx[nx] = gc[nx - 1]
    sy = np.empty((nx, ny + 1))
    sy[:, 0] = gc[:, 0]
    sy[:, 1:ny] = 0.5 * (gc[:, :-1] + gc[:, 1:])
    sy[:, ny] = gc[:, ny - 1]
    return {"grav_coeff": np.asfortranarray(gc), "d_grav_coeff_dx": np.asfortranarray(dgc),
            "grav_coeff_stag_x": np.asfortranarray(sx), "grav_coeff_stag_y": np.asfortranarray(sy)}


def init_radial_source(p, x_source, y_source, r_source):
    """Inlet cells of a circular radial source: init_source
    (src/geometry_2d.f90:872-1102, radial branch).  Returns the planes
    source_cell, sourceE/W/S/N and source*_vect_x/y."""
    nx, ny = p.nx, p.ny
    x_stag, x_comp, y_stag, y_comp = grid(p)
    sc = np.zeros((nx, ny), np.int32)
    flags = {s: np.zeros((nx, ny), np.int8) for s in "EWSN"}
    vx = {s: np.zeros((nx, ny)) for s in "EWSN"}
    vy = {s: np.zeros((nx, ny)) for s in "EWSN"}
    r2 = r_source ** 2
    dx = x_stag[1] - x_stag[0]
    pad = int(math.ceil(r_source / dx)) + 3
    j0 = max(2, int((x_source - p.x0) / dx) - pad)
    j1 = min(nx - 1, int((x_source - p.x0) / dx) + pad)
    dy = y_stag[1] - y_stag[0]
    k0 = max(2, int((y_source - p.y0) / dy) - pad)
    k1 = min(ny - 1, int((y_source - p.y0) / dy) + pad)
    for k in range(k0, k1 + 1):            # 1-based Fortran indices
        for j in range(j0, j1 + 1):
            xc, yc = x_comp[j - 1], y_comp[k - 1]
            if (xc - x_source) ** 2 + (yc - y_source) ** 2 <= r2:
                sc[j - 1, k - 1] = 1
                if (x_comp[j - 2] - x_source) ** 2 + (yc - y_source) ** 2 >= r2:
                    sc[j - 2, k - 1] = 2
                    flags["E"][j - 2, k - 1] = 1
                    d = math.sqrt((x_stag[j - 1] - x_source) ** 2 + (yc - y_source) ** 2)
                    vx["E"][j - 2, k - 1] = (x_stag[j - 1] - x_source) * r_source / d ** 2
                    vy["E"][j - 2, k - 1] = (yc - y_source) * r_source / d ** 2
                elif (x_comp[j] - x_source) ** 2 + (yc - y_source) ** 2 >= r2:
                    sc[j, k - 1] = 2
                    flags["W"][j, k - 1] = 1
                    d = math.sqrt((x_stag[j] - x_source) ** 2 + (yc - y_source) ** 2)
                    vx["W"][j, k - 1] = (x_stag[j] - x_source) * r_source / d ** 2
                    vy["W"][j, k - 1] = (yc - y_source) * r_source / d ** 2
                if (xc - x_source) ** 2 + (y_comp[k - 2] - y_source) ** 2 >= r2:
                    sc[j - 1, k - 2] = 2
                    flags["N"][j - 1, k - 2] = 1
                    d = math.sqrt((xc - x_source) ** 2 + (y_stag[k - 1] - y_source) ** 2)
                    vx["N"][j - 1, k - 2] = (xc - x_source) * r_source / d ** 2
                    vy["N"][j - 1, k - 2] = (y_stag[k - 1] - y_source) * r_source / d ** 2
                elif (xc - x_source) ** 2 + (y_comp[k] - y_source) ** 2 >= r2:
                    sc[j - 1, k] = 2
                    flags["S"][j - 1, k] = 1
                    d = math.sqrt((xc - x_source) ** 2 + (y_stag[k] - y_source) ** 2)
                    vx["S"][j - 1, k] = (xc - x_source) * r_source / d ** 2
                    vy["S"][j - 1, k] = (y_stag[k] - y_source) * r_source / d ** 2
    out = {"source_cell": sc}
    for s in "EWSN":
        out["source" + s] = flags[s]
        out["source%s_vect_x" % s] = vx[s]
        out["source%s_vect_y" % s] = vy[s]
    return out


def mixt_rho_m_red_grav(p, qp):
    """mixt_var (constitutive_2d.f90:1333-1483) for one physical state."""
    ns = p.n_solid
    h = qp[0]
    if h <= EPSILON:
        return p.pres / (p.sp_gas_const_a * p.T_ambient), 0.0
    T = qp[3]
    al = [qp[4 + i] if p.alpha_flag else qp[4 + i] / h for i in range(ns)]
    at = sum(al)
    rho_a = p.pres / (p.sp_gas_const_a * T)
    rho_c = (((1.0 - 0.0) - at) - 0.0) * rho_a / ((1.0 - 0.0) - at)
    rho_m = (1.0 - at) * rho_c + sum(al[i] * p.rho_s[i] for i in range(ns))
    rho_a_amb = p.pres / (p.sp_gas_const_a * p.T_ambient)
    return rho_m, (rho_m - rho_a_amb) / rho_m * p.grav


def set_radial_source_state(p, r_source, mfr_source, vel_source, T_source, xs_source):
    """Inlet thickness, velocity and solid volume fractions from the mass
    flow rate and velocity (src/inpout_2d.f90:4250-4500, MFR + VEL branch)."""
    ns = p.n_solid
    source_length = math.pi * (r_source + r_source) * 1.0
    xs_tot = sum(xs_source)
    xc = 1.0 - xs_tot
    inv_pres = 1.0 / p.pres
    sgc = ((xc - 0.0) * p.sp_gas_const_a + 0.0) / xc
    inv_rho_c = sgc * T_source * inv_pres
    inv_rhom = sum(xs_source[i] * (1.0 / p.rho_s[i]) for i in range(ns)) + xc * inv_rho_c
    rho_m = 1.0 / inv_rhom
    alphas = [rho_m * xs_source[i] * (1.0 / p.rho_s[i]) for i in range(ns)]
    h = 1.0
    qp = [h, h * vel_source, 0.0, T_source] + [a * h for a in alphas] + [vel_source, 0.0]
    rho_m2, _ = mixt_rho_m_red_grav(p, qp)
    h_source = mfr_source / (source_length * rho_m2 * vel_source * 1.0)
    p.h_source = h_source
    p.vel_source = vel_source
    p.T_source = T_source
    for i in range(ns):
        p.alphas_source[i] = alphas[i]
    p.radial_source_flag = 1
    return h_source


def qp_to_qc_grid(p, qp):
    """Vectorised qp_to_qc (constitutive_2d.f90:1709-2140) for building
    initial states; qp is (n_vars+2, nx, ny)."""
    ns = p.n_solid
    nv = 4 + ns
    h = qp[0]
    wet = h > EPSILON
    hs = np.where(wet, h, 1.0)
    T = np.where(wet, qp[3], p.T_ambient)
    al = [qp[4 + i] if p.alpha_flag else qp[4 + i] / hs for i in range(ns)]
    at = sum(al)
    rho_a = p.pres / (p.sp_gas_const_a * T)
    rho_c = ((1.0 - at) * rho_a) / (1.0 - at)
    rho_m = (1.0 - at) * rho_c + sum(al[i] * p.rho_s[i] for i in range(ns))
    xs = [al[i] * p.rho_s[i] / rho_m for i in range(ns)]
    xc = (1.0 - at) * rho_c / rho_m
    cpm = sum(xs[i] * p.sp_heat_s[i] for i in range(ns)) + xc * p.sp_heat_a
    u, v = qp[nv], qp[nv + 1]
    qc = np.zeros((nv,) + h.shape)
    qc[0] = rho_m * h
    qc[1] = rho_m * qp[1]
    qc[2] = rho_m * qp[2]
    if p.energy_flag:
        qc[3] = h * rho_m * (cpm * T + 0.5 * (u * u + v * v))
    else:
        qc[3] = h * rho_m * cpm * T
    for i in range(ns):
        qc[4 + i] = xs[i] * qc[0]
    qc[:, ~wet] = 0.0
    return np.asfortranarray(qc)


def fractal_dem(n, dx, hurst, relief, slope_deg, seed):
    """Seeded spectral-synthesis surface: power spectrum ~ k^-(2H+2), rescaled
    to `relief` metres of range, plus a planar tilt of `slope_deg` degrees
    descending in +x.  Returns (n, n) float64 indexed [j, k]."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n)
    ky = np.fft.rfftfreq(n)
    K = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    K[0, 0] = 1.0
    amp = K ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * phase)
    z = np.fft.irfft2(spec, s=(n, n))
    z = (z - z.min()) / (z.max() - z.min()) * relief
    x = np.arange(n) * dx
    tilt = -math.tan(math.radians(slope_deg)) * x
    B = z + tilt[:, None]
    return np.asfortranarray(B - B.min())


# --------------------------------------------------------------- workloads

def dambreak(nx=200, ny=200, dx=0.05, h_left=1.0, h_right=0.1, x_split=5.0,
             alpha=0.01, T=300.0, rheology=None):
    """Plain method, 2-D dam break on a flat bed (first workload: 200x200
    cells of 0.05 m, 1 solid class d=1e-4 m, rho_s=2500, volume fraction
    0.01, T=300 K, minmod, CFL 0.24, 2-stage IMEX RK, transmissive)."""
    p = default_params(nx, ny, 1, dx)
    p.rho_s[0] = 2500.0
    p.diam_s[0] = 1.0e-4
    p.sp_heat_s[0] = 1617.0
    p.max_dt = 1.0e-2
    transmissive_bcs(p)
    if rheology is not None:
        p.rheology_flag = 1
        p.rheology_model = rheology
        if rheology == 1:
            p.mu, p.xi = 0.1, 500.0
        elif rheology == 6:
            p.friction_factor = 1.0e-3
    _, x_comp, _, y_comp = grid(p)
    X = np.repeat(x_comp[:, None], ny, axis=1)
    h = np.where(X < x_split, h_left, h_right)
    nv = 5
    qp = np.zeros((nv + 2, nx, ny))
    qp[0] = h
    qp[3] = T
    qp[4] = alpha * h
    q = qp_to_qc_grid(p, qp)
    zeros = np.zeros((nx, ny))
    static = {"B_cent": zeros, "B_prime_x_geom": zeros, "B_prime_y_geom": zeros,
              "solve_mask_time": zeros}
    return p, static, q


def radial_current(nx=1024, ny=1024, dx=2.0, bump_h=20.0, bump_sigma=200.0,
                   r_source=20.0, mfr=5.0e6, T_source=900.0, vel_source=10.0,
                   xs=(0.57, 0.38), diam=(1.0e-4, 1.0e-3), mu=0.1, xi=500.0):
    """Plain method, radial gas-particle current over a Gaussian bump (second
    workload: 1024^2 cells of 2 m, circular inlet r=20 m at 5e6 kg/s, T=900 K,
    two solid classes split 0.6/0.4 of the solid mass, Voellmy mu=0.1 xi=500).
    The inlet carries 95% solid by mass (the split of the two classes is
    0.6/0.4); VEL_SOURCE = 10 m/s.  Every boundary variable is zero-gradient,
    the boundary set of the reference's ensemble example for radial
    currents (zero_gradient_bcs); under the dam-break set (h extrapolated by
    its one-sided slope) the 510 m thick current breaks down where it
    reaches the border."""
    ns = len(xs)
    p = default_params(nx, ny, ns, dx)
    for i in range(ns):
        p.rho_s[i] = 2500.0
        p.diam_s[i] = diam[i]
        p.sp_heat_s[i] = 1617.0
    p.rheology_flag = 1
    p.rheology_model = 1
    p.mu, p.xi = mu, xi
    p.max_dt = 1.0
    zero_gradient_bcs(p)
    _, x_comp, _, y_comp = grid(p)
    xs0 = x_comp[nx // 2]
    ys0 = y_comp[ny // 2]
    X, Y = np.meshgrid(x_comp, y_comp, indexing="ij")
    r2 = (X - xs0) ** 2 + (Y - ys0) ** 2
    B = np.asfortranarray(bump_h * np.exp(-r2 / (2.0 * bump_sigma ** 2)))
    static = {"B_cent": B, "solve_mask_time": np.zeros((nx, ny))}
    static.update(topography_geom(B, p.cell_size, p.cell_size))
    # inlet centre a fraction of a cell off the cell centres, so that no cell
    # centre lies exactly on the inlet circle
    src_x = xs0 - 0.25 * nx * dx + 0.31 * dx
    src_y = ys0 + 0.17 * dx
    static.update(init_radial_source(p, src_x, src_y, r_source))
    set_radial_source_state(p, r_source, mfr, vel_source, T_source, list(xs))
    q = np.zeros((4 + ns, nx, ny), order="F")
    return p, static, q


def fractal_inlet(n=4096, dx=10.0, hurst=0.8, relief=800.0, slope_deg=15.0,
                  seed=20261203, mfr=1.0e7, T_source=1000.0, vel_source=20.0,
                  r_source=50.0, xs=(0.3, 0.3, 0.35), diam=(1.0e-5, 1.0e-4, 1.0e-3),
                  erosion_coeff=1.0e-4, erodible_thickness=1.0, initial_layer=0.0,
                  layer_alpha=0.02, mu=0.1, xi=500.0):
    """Plain method at scale on a synthetic fractal DEM (third workload:
    4096^2 cells of 10 m, Hurst 0.8, 800 m relief plus a 15 degree mean slope,
    seeded; inlet 1e7 kg/s at 1000 K; three solid classes 1e-5/1e-4/1e-3 m
    with settling and erosion of a 1 m erodible layer).  `initial_layer` > 0
    covers the whole DEM with a resting current of that thickness (used by
    the throughput benchmark so that every cell carries the full physics)."""
    ns = len(xs)
    p = default_params(n, n, ns, dx)
    for i in range(ns):
        p.rho_s[i] = 2500.0
        p.diam_s[i] = diam[i]
        p.sp_heat_s[i] = 1617.0
    p.rheology_flag = 1
    p.rheology_model = 1
    p.mu, p.xi = mu, xi
    p.max_dt = 1.0
    p.settling_flag = 1
    p.erosion_coeff = erosion_coeff
    p.erodible_porosity = 0.4
    p.coeff_porosity = p.erodible_porosity / (1.0 - p.erodible_porosity)
    p.T_erodible = 300.0
    p.rho_c_sub = p.pres / (p.sp_gas_const_a * p.T_erodible)
    for i in range(ns):
        p.erodible_fract[i] = 1.0 / ns
    transmissive_bcs(p)
    B = fractal_dem(n, dx, hurst, relief, slope_deg, seed)
    static = {"B_cent": B, "solve_mask_time": np.zeros((n, n))}
    static.update(topography_geom(B, dx, dx))
    _, x_comp, _, y_comp = grid(p)
    src_x = x_comp[max(8, n // 8)] + 0.31 * dx
    src_y = y_comp[n // 2] + 0.17 * dx
    static.update(init_radial_source(p, src_x, src_y, r_source))
    set_radial_source_state(p, r_source, mfr, vel_source, T_source, list(xs))
    er = np.zeros((ns, n, n), order="F")
    for i in range(ns):
        er[i] = p.erodible_fract[i] * (1.0 - p.erodible_porosity) * erodible_thickness
    static["erodible"] = er
    static["deposit"] = np.zeros((n, n, ns), order="F")
    static["erosion"] = np.zeros((n, n, ns), order="F")
    if initial_layer > 0.0:
        nv = 4 + ns
        qp = np.zeros((nv + 2, 1, 1))
        qp[0] = initial_layer
        qp[3] = T_source
        for i in range(ns):
            qp[4 + i] = layer_alpha / ns * initial_layer
        cell = qp_to_qc_grid(p, qp)[:, 0, 0]   # the layer is uniform
        q = np.empty((nv, n, n), order="F")
        for i in range(nv):
            q[i] = cell[i]
        q[:, static["source_cell"] == 1] = 0.0
    else:
        q = np.zeros((4 + ns, n, n), order="F")
    return p, static, q


def ensemble_members(n_members=256, side_min=256, side_max=1024, dx=2.0, seed=20261204,
                     bump_h=(5.0, 50.0), bump_sigma=(50.0, 300.0), mfr=(1.0e6, 1.0e8),
                     T_source=(600.0, 1200.0), diam=(1.0e-5, 1.0e-3), r_source=20.0,
                     bcs="ensemble"):
    """Batched-ensemble workload (fourth workload): members on their own
    square grids of 2 m cells, side uniform in [side_min, side_max]; a
    Gaussian bump of uniform random height and sigma; a radial inlet of
    r = 20 m with log-uniform mass flow, uniform temperature and one solid
    class of log-uniform diameter (95% solid by mass, Voellmy friction as in
    the radial-current workload).  The sampling follows the reference's
    ensemble example (EXAMPLES/EXAMPLE_ENSEMBLE_ETNA/create_ensemble.py:35-55:
    log-uniform and uniform 1-D sampling), and so do the boundaries: every
    variable zero-gradient (bcs="ensemble"); bcs="dambreak" keeps the
    radial-current workload's TEST_DAMBREAK set (h extrapolated by the
    one-sided slope), under which thick currents that reach the border
    break down.  Returns a list of (params, static, q, sample) with `sample`
    the drawn values."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_members):
        side = int(rng.integers(side_min, side_max + 1))
        s = {"side": side,
             "bump_h": float(rng.uniform(*bump_h)),
             "bump_sigma": float(rng.uniform(*bump_sigma)),
             "mfr": float(10.0 ** rng.uniform(np.log10(mfr[0]), np.log10(mfr[1]))),
             "T_source": float(rng.uniform(*T_source)),
             "diam": float(10.0 ** rng.uniform(np.log10(diam[0]), np.log10(diam[1])))}
        p, st, q = radial_current(nx=side, ny=side, dx=dx, bump_h=s["bump_h"],
                                  bump_sigma=s["bump_sigma"], r_source=r_source, mfr=s["mfr"],
                                  T_source=s["T_source"], xs=(0.95,), diam=(s["diam"],))
        if bcs == "dambreak":
            transmissive_bcs(p)
        out.append((p, st, q, s))
    return out
